"""Independent numpy restatements of the matrix variant of the JST
dissipation (makeArtificialDissipation2 with useMatrixDissipation,
def_par:11513-11906: the undivided Laplacian with dE + dp, the pressure
sensor, and the one-dimensional Roe matrix |A| with Harten's correction
applied to the Laplacian and state differences) and of dissipation scheme 1,
checked against the CPU restatement's dissipation at the same state."""
import ctypes

import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

GAM = 1.4


@pytest.mark.parametrize("harten", [0.0, 0.3])
def test_numpy_matrix_dissipation_matches_the_restatement(harten):
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=1)
    k2, k4 = 0.6, 0.2
    c = default_controls(ReynoldsNumber=0.0, fluxType=1, numberOfGridsToUse=1, useMatrixDissipation=1,
                         HartensCorrectionFactor=harten, secondOrderDissipationFactor=k2,
                         fourthOrderDissipationFactor=k4)
    u = initial_state(c, mesh, perturb_seed=9, amplitude=0.05)
    N = u.shape[1]
    u[1] *= 1.0 + 0.03 * np.sin(np.arange(N))
    u[4] *= 1.0 + 0.01 * np.cos(0.3 * np.arange(N))
    u = np.ascontiguousarray(u)
    o = Solver(c, mesh, backend=oracle_backend())
    diss = np.zeros((5, N))
    p_ = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    assert o.be.dissipation(o._h, 1, p_(u), p_(diss)) == 0

    i1, i2 = mesh.array(1, "side_idx") - 1
    w = mesh.array(1, "side_w")
    p = np.abs(np.maximum((GAM - 1) * (u[4] - 0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / u[0]), 0.1))
    conn = np.zeros(N)
    np.add.at(conn, i1, 1.0)
    np.add.at(conn, i2, 1.0)
    lap = np.zeros((5, N))
    d = u[:, i1] - u[:, i2]
    d[4] = d[4] + p[i1] - p[i2]
    for k in range(5):
        np.add.at(lap[k], i1, -d[k])
        np.add.at(lap[k], i2, d[k])
    lap /= conn
    s7, s8 = np.zeros(N), np.zeros(N)
    np.add.at(s7, i1, -(p[i1] - p[i2]))
    np.add.at(s7, i2, p[i1] - p[i2])
    np.add.at(s8, i1, p[i1] + p[i2])
    np.add.at(s8, i2, p[i1] + p[i2])
    sens = 12.0 * np.abs(s7 / s8)

    g1 = GAM - 1.0
    al = np.sqrt((w ** 2).sum(0))
    n = w / al
    rl, rr = u[0, i1], u[0, i2]
    vl, vr = u[1:4, i1] / rl, u[1:4, i2] / rr
    hl, hr = (u[4, i1] + p[i1]) / rl, (u[4, i2] + p[i2]) / rr
    di = np.sqrt(rr / rl)
    d1 = 1.0 / (di + 1.0)
    vi = (di * vr + vl) * d1
    hi = (di * hr + hl) * d1
    af = 0.5 * (vi ** 2).sum(0)
    ci2 = g1 * (hi - af)
    ci = np.sqrt(ci2)
    ucp = (vi * n).sum(0)
    lam = [np.abs(ucp + ci), np.abs(ucp - ci), np.abs(ucp)]
    eps1 = 1.0 / max(harten, 1e-5)
    lam = [np.where(x < harten, 0.5 * (x * x * eps1 + harten), x) for x in lam]
    s1, s2, l3 = 0.5 * (lam[0] + lam[1]), 0.5 * (lam[0] - lam[1]), lam[2]

    def absA(dv):
        a1 = g1 * (af * dv[0] - (vi * dv[1:4]).sum(0) + dv[4])
        a2 = -ucp * dv[0] + (dv[1:4] * n).sum(0)
        c1 = (s1 - l3) * a1 / ci2 + s2 * a2 / ci
        c2 = s2 * a1 / ci + (s1 - l3) * a2
        return al * np.concatenate([[l3 * dv[0] + c1], l3 * dv[1:4] + c1 * vi + c2 * n,
                                    [l3 * dv[4] + c1 * hi + c2 * ucp]])

    d4v = absA(lap[:, i1] - lap[:, i2])
    d2v = absA(u[:, i1] - u[:, i2])
    dd2 = k2 * np.maximum(sens[i1], sens[i2])
    dd4 = np.maximum(k4 - dd2, 0.0)
    ref = np.zeros((5, N))
    for k in range(5):
        t = -d4v[k] * dd4 + d2v[k] * dd2
        np.add.at(ref[k], i1, t)
        np.add.at(ref[k], i2, -t)
    scale = np.abs(ref).max(axis=1, keepdims=True)
    assert np.all(scale > 0)
    np.testing.assert_allclose(diss / scale, ref / scale, rtol=0, atol=1e-11)


def test_numpy_scheme1_dissipation_matches_the_restatement():
    # makeArtificialDissipation1 (def_par:10706-11482) with its default
    # (matrix) branch: L^ = L(U) + grad U . L(x) (as coded), L(x) = 0 on
    # boundary nodes, the same pressure sensor and Roe matrix as above
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=1)
    k2, k4 = 0.5, 0.05
    c = default_controls(ReynoldsNumber=0.0, fluxType=1, numberOfGridsToUse=1, dissipationScheme=1,
                         secondOrderDissipationFactor=k2, fourthOrderDissipationFactor=k4)
    u = initial_state(c, mesh, perturb_seed=9, amplitude=0.05)
    N = u.shape[1]
    Nb = mesh.level(1).n_bnodes
    u[1] *= 1.0 + 0.03 * np.sin(np.arange(N))
    u = np.ascontiguousarray(u)
    o = Solver(c, mesh, backend=oracle_backend())
    diss = np.zeros((5, N))
    p_ = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    assert o.be.dissipation(o._h, 1, p_(u), p_(diss)) == 0

    i1, i2 = mesh.array(1, "side_idx") - 1
    b1, b2 = mesh.array(1, "bnd_idx")[:2] - 1
    w, bw = mesh.array(1, "side_w"), mesh.array(1, "bnd_w")
    V, x = mesh.array(1, "volume"), mesh.array(1, "coords")
    p = np.abs(np.maximum((GAM - 1) * (u[4] - 0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / u[0]), 0.1))
    grad = np.zeros((3, 5, N))
    for a in range(3):
        s = (u[:, i1] + u[:, i2]) * w[a]
        for k in range(5):
            np.add.at(grad[a, k], i1, s[k])
            np.add.at(grad[a, k], i2, -s[k])
            np.add.at(grad[a, k], b1, (3 * u[k, b1] + u[k, b2]) * bw[a])
            np.add.at(grad[a, k], b2, (u[k, b1] + 3 * u[k, b2]) * bw[a])
    grad /= V
    lu, lx = np.zeros((5, N)), np.zeros((3, N))
    for k in range(5):
        np.add.at(lu[k], i1, -(u[k, i1] - u[k, i2]))
        np.add.at(lu[k], i2, u[k, i1] - u[k, i2])
    for a in range(3):
        np.add.at(lx[a], i1, -(x[a, i1] - x[a, i2]))
        np.add.at(lx[a], i2, x[a, i1] - x[a, i2])
    lx[:, :Nb] = 0.0
    lhat = lu + np.einsum("akn,an->kn", grad, lx)
    s7, s8 = np.zeros(N), np.zeros(N)
    np.add.at(s7, i1, -(p[i1] - p[i2]))
    np.add.at(s7, i2, p[i1] - p[i2])
    np.add.at(s8, i1, p[i1] + p[i2])
    np.add.at(s8, i2, p[i1] + p[i2])
    sens = 12.0 * np.abs(s7 / s8)

    g1 = GAM - 1.0
    al = np.sqrt((w ** 2).sum(0))
    n = w / al
    rl, rr = u[0, i1], u[0, i2]
    vl, vr = u[1:4, i1] / rl, u[1:4, i2] / rr
    hl, hr = (u[4, i1] + p[i1]) / rl, (u[4, i2] + p[i2]) / rr
    di = np.sqrt(rr / rl)
    d1 = 1.0 / (di + 1.0)
    vi = (di * vr + vl) * d1
    hi = (di * hr + hl) * d1
    af = 0.5 * (vi ** 2).sum(0)
    ci2 = g1 * (hi - af)
    ci = np.sqrt(ci2)
    ucp = (vi * n).sum(0)
    l1, l2, l3 = np.abs(ucp + ci), np.abs(ucp - ci), np.abs(ucp)
    s1, s2 = 0.5 * (l1 + l2), 0.5 * (l1 - l2)

    def absA(dv):
        a1 = g1 * (af * dv[0] - (vi * dv[1:4]).sum(0) + dv[4])
        a2 = -ucp * dv[0] + (dv[1:4] * n).sum(0)
        c1 = (s1 - l3) * a1 / ci2 + s2 * a2 / ci
        c2 = s2 * a1 / ci + (s1 - l3) * a2
        return al * np.concatenate([[l3 * dv[0] + c1], l3 * dv[1:4] + c1 * vi + c2 * n,
                                    [l3 * dv[4] + c1 * hi + c2 * ucp]])

    d4v = absA(lhat[:, i1] - lhat[:, i2])
    d2v = absA(u[:, i1] - u[:, i2])
    dd2 = k2 * np.maximum(sens[i1], sens[i2])
    dd4 = np.maximum(k4 - dd2, 0.0)
    ref = np.zeros((5, N))
    for k in range(5):
        t = -d4v[k] * dd4 + d2v[k] * dd2
        np.add.at(ref[k], i1, t)
        np.add.at(ref[k], i2, -t)
    scale = np.abs(ref).max(axis=1, keepdims=True)
    np.testing.assert_allclose(diss / scale, ref / scale, rtol=0, atol=1e-11)
