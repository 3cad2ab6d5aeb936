"""An independent numpy restatement of the upwind extension's level-1 edge
flux (the Roe flux of MUSCL / Van Albada states from the Galerkin gradients,
with the upwind sign), checked against the CPU restatement through the
difference of two residuals: the boundary fluxes of fluxType 3 are the same
with and without the extension, so R(extension) - R(reference Roe) is the
edge sum of f(extension) - f(reference Roe)."""
import numpy as np

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

GAM = 1.4


def roe(ra, ua, va, wa, Ea, pa, rb, ub, vb, wb, Eb, pb, w, upwind):
    g1 = GAM - 1.0
    rnorm = np.sqrt((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2])
    n = w / rnorm
    rua, rva, rwa, rha = ra * ua, ra * va, ra * wa, Ea + pa
    rub, rvb, rwb, rhb = rb * ub, rb * vb, rb * wb, Eb + pb
    nva = ua * n[0] + va * n[1] + wa * n[2]
    nvb = ub * n[0] + vb * n[1] + wb * n[2]
    di = np.sqrt(ra / rb)
    d1 = 1.0 / (di + 1.0)
    ui, vi, wi = (di * ua + ub) * d1, (di * va + vb) * d1, (di * wa + wb) * d1
    hi = (di * rha / ra + rhb / rb) * d1
    af = 0.5 * (ui * ui + vi * vi + wi * wi)
    ci2 = np.maximum(g1 * (hi - af), 1e-5)
    ci = np.sqrt(ci2)
    ucp = ui * n[0] + vi * n[1] + wi * n[2]
    s = 1.0 if upwind else -1.0  # du = q2 - q1 (upwind) or q1 - q2 (the reference)
    du = s * np.array([rb - ra, rub - rua, rvb - rva, rwb - rwa, Eb - Ea])
    l1, l2, l3 = np.abs(ucp + ci), np.abs(ucp - ci), np.abs(ucp)
    s1, s2 = 0.5 * (l1 + l2), 0.5 * (l1 - l2)
    al1 = g1 * (af * du[0] - ui * du[1] - vi * du[2] - wi * du[3] + du[4])
    al2 = -ucp * du[0] + du[1] * n[0] + du[2] * n[1] + du[3] * n[2]
    c1 = (s1 - l3) * al1 / ci2 + s2 * al2 / ci
    c2 = s2 * al1 / ci + (s1 - l3) * al2
    F = np.array([ra * nva + rb * nvb,
                  pa * n[0] + rua * nva + pb * n[0] + rub * nvb,
                  pa * n[1] + rva * nva + pb * n[1] + rvb * nvb,
                  pa * n[2] + rwa * nva + pb * n[2] + rwb * nvb,
                  rha * nva + rhb * nvb])
    D = np.array([l3 * du[0] + c1, l3 * du[1] + c1 * ui + c2 * n[0], l3 * du[2] + c1 * vi + c2 * n[1],
                  l3 * du[3] + c1 * wi + c2 * n[2], l3 * du[4] + c1 * hi + c2 * ucp])
    return rnorm * (F - D)


def test_numpy_extension_flux_matches_the_restatement():
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=1)
    base = dict(ReynoldsNumber=0.0, fluxType=3, numberOfGridsToUse=1)
    c_ext = default_controls(**base, reconstruction=1)
    c_ref = default_controls(**base)
    u = initial_state(c_ext, mesh, perturb_seed=7, amplitude=0.05)
    N = u.shape[1]
    u[1] *= 1.0 + 0.02 * np.sin(np.arange(N))
    u[3] += 0.01 * np.cos(0.7 * np.arange(N))
    r_ext = Solver(c_ext, mesh, backend=oracle_backend()).residual_fwd(u)
    r_ref = Solver(c_ref, mesh, backend=oracle_backend()).residual_fwd(u)

    idx = mesh.array(1, "side_idx") - 1
    w = mesh.array(1, "side_w")
    bidx = mesh.array(1, "bnd_idx")[:2] - 1
    bw = mesh.array(1, "bnd_w")
    V = mesh.array(1, "volume")
    x = mesh.array(1, "coords")
    q = np.array([u[0], u[1] / u[0], u[2] / u[0], u[3] / u[0], u[4]])
    # Galerkin gradient (interior edges, then boundary edges with 2 q_own + q1 + q2)
    g = np.zeros((3, 5, N))
    for a in range(3):
        s = (q[:, idx[0]] + q[:, idx[1]]) * w[a]
        for k in range(5):
            np.add.at(g[a, k], idx[0], s[k])
            np.add.at(g[a, k], idx[1], -s[k])
        sb = q[:, bidx[0]] + q[:, bidx[1]]
        for k in range(5):
            np.add.at(g[a, k], bidx[0], (2 * q[k, bidx[0]] + sb[k]) * bw[a])
            np.add.at(g[a, k], bidx[1], (2 * q[k, bidx[1]] + sb[k]) * bw[a])
    g /= V
    i1, i2 = idx
    d = x[:, i2] - x[:, i1]
    q1, q2 = q[:, i1], q[:, i2]
    dq = q2 - q1
    g1 = np.einsum("akn,an->kn", g[:, :, i1], d)
    g2 = np.einsum("akn,an->kn", g[:, :, i2], d)

    def va(a, b):
        ab = a * b
        return np.where(ab > 0, ab * (a + b) / np.where(ab > 0, a * a + b * b, 1.0), 0.0)

    qa = q1 + 0.5 * va(2 * g1 - dq, dq)
    qb = q2 - 0.5 * va(2 * g2 - dq, dq)
    pres = lambda s: (GAM - 1) * (s[4] - 0.5 * (s[1] ** 2 + s[2] ** 2 + s[3] ** 2) * s[0])
    pa, pb = pres(qa), pres(qb)
    ok = (qa[0] > 0) & (qb[0] > 0) & (pa > 0) & (pb > 0)
    qa, qb = np.where(ok, qa, q1), np.where(ok, qb, q2)
    pa, pb = pres(qa), pres(qb)
    f_ext = roe(*qa, pa, *qb, pb, w, upwind=True)
    # the reference's Roe branch on the node states, with the pressure floor
    p = np.maximum((GAM - 1) * (u[4] - 0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / u[0]), 0.1)
    f_ref = roe(u[0, i1], u[1, i1] / u[0, i1], u[2, i1] / u[0, i1], u[3, i1] / u[0, i1], u[4, i1], p[i1],
                u[0, i2], u[1, i2] / u[0, i2], u[2, i2] / u[0, i2], u[3, i2] / u[0, i2], u[4, i2], p[i2],
                w, upwind=False)
    diff = np.zeros((5, N))
    for k in range(5):
        np.add.at(diff[k], i1, f_ext[k] - f_ref[k])
        np.add.at(diff[k], i2, -(f_ext[k] - f_ref[k]))
    scale = np.abs(r_ext).max(axis=1, keepdims=True)
    assert ok.mean() > 0.9
    np.testing.assert_allclose((r_ext - r_ref) / scale, diff / scale, rtol=0, atol=1e-11)
