"""Independent numpy restatements of the benchmark workload's own terms.

Written from the Fortran (SolverSource/mgnsg3d_def_par.F90), not from the
CPU restatement in oracle/, and checked against that restatement at the same
state on a jittered bump-channel mesh:

* makePressureField (:13612-13630) and makeTimeSteps (:13335-13610): the
  inviscid spectral radius |v.w| + c|w| per interior edge and the doubled
  boundary-face terms, the viscous 2 max(1/Re, mu) |w|^2 / rho (the other
  node's on interior edges), dt = 0.5 / (sum/V + visc/V^2);
* makeArtificialDissipation2, scalar branch (:11484-11993): the undivided
  Laplacian with dE + dp over the connectivity, the pressure sensor
  12 |sum dp / sum p|, d0 = min(V/dt)/(n1 + n2), d2 = d0 k2 max(sensor),
  d4 = dim(d0 k4, d2); with and without useDissipationWeighting;
* makeViscosityTerm (:5198-5893): Galerkin gradients of (u, v, w, T) with
  the boundary-face terms, Sutherland's viscosity, the stress tensor and heat
  flux, the adiabatic-wall projection (setTemperatureForAdiabaticWall
  :5170-5196), the wall stress, and the edge and boundary-face fluxes;
* makeRHS for the central flux (:1664-1669, 2089-2100) with the wall and
  far-field (Roe against the freestream) boundary faces (:2182-2446);
* one smoother iteration of level 1 (singleIteration :1002-1181 with
  solveSystem :1407-1479, updateSolutionVector :1292-1405 and limitDensity
  :1243-1257): three stages with 0.6, 0.6, 1, compared at the nodes three or
  more edges away from every boundary node, which no boundary condition
  reaches within three stages.

Tolerance: 1e-11 relative to each component's largest magnitude (numpy sums
in another order than the reference's edge loop).
"""
import ctypes

import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

TOL = 1e-11


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class Geo:
    """Level-1 arrays of a jittered bump channel (side and boundary
    coefficients and volumes recomputed at the moved coordinates)."""

    def __init__(self, nx, ny, nz, seed=3):
        base = Mesh.bump_channel(nx, ny, nz, 0.05, nlevels=1)
        X = base.array(1, "coords")
        nb = base.level(1).n_bnodes
        jit = np.random.default_rng(seed).uniform(-1, 1, X.shape) * 0.12 / nz
        jit[:, :nb] = 0.0
        self.X = X + jit
        self.sw, self.bw, self.V = base.geometry(self.X)
        self.mesh = base.with_level1_geometry(self.sw, self.bw, self.V)
        self.base = base
        self.i1, self.i2 = base.array(1, "side_idx") - 1
        bidx = base.array(1, "bnd_idx")
        self.b1, self.b2, self.bind = bidx[0] - 1, bidx[1] - 1, bidx[2]
        self.slen = base.array(1, "side_len")
        self.N, self.Nb = base.level(1).n_nodes, nb
        reg, ind = base.array(1, "node_reg"), base.array(1, "node_ind")
        self.wall = ind[reg[0] - 1:reg[1]] - 1
        self.bnodes = ind[:nb] - 1
        self.conn = np.zeros(self.N)
        np.add.at(self.conn, self.i1, 1.0)
        np.add.at(self.conn, self.i2, 1.0)
        # makeBoundaryNormals (def_par:15394-15521): n = -sum w_b / |.|
        a = np.zeros((3, self.N))
        for k in range(3):
            np.add.at(a[k], self.b1, -self.bw[k])
            np.add.at(a[k], self.b2, -self.bw[k])
        nrm = np.sqrt((a ** 2).sum(0))
        self.normal = np.where(nrm > 1e-10, a / np.where(nrm > 1e-10, nrm, 1.0), 0.0)


def pressure(c, u):
    p = (c.gamma - 1.0) * (u[4] - 0.5 * (u[1] ** 2 + u[2] ** 2 + u[3] ** 2) / u[0])
    return np.maximum(p, 0.1)


def time_steps(c, g, u, p, mu):
    i1, i2, b1, b2 = g.i1, g.i2, g.b1, g.b2
    dt = np.zeros(g.N)
    visc = np.zeros(g.N)
    w = g.sw
    al = (w ** 2).sum(0)
    cc1 = np.maximum(c.gamma * p[i1] / u[0, i1], 0.001)
    cc2 = np.maximum(c.gamma * p[i2] / u[0, i2], 0.001)
    vn1 = (w * u[1:4, i1]).sum(0) / u[0, i1]
    vn2 = (w * u[1:4, i2]).sum(0) / u[0, i2]
    np.add.at(dt, i1, np.abs(vn1) + np.sqrt(cc1 * al))
    np.add.at(dt, i2, np.abs(vn2) + np.sqrt(cc2 * al))
    am = 1.0 / c.ReynoldsNumber if c.ReynoldsNumber > 0 else 0.0
    if c.ReynoldsNumber > 0:
        dv1 = 2.0 * np.maximum(am, mu[i1]) * al / u[0, i1]
        dv2 = 2.0 * np.maximum(am, mu[i2]) * al / u[0, i2]
        np.add.at(visc, i1, dv2)
        np.add.at(visc, i2, dv1)
    bw = g.bw
    al = (bw ** 2).sum(0)
    cc1 = np.sqrt(np.maximum(c.gamma * p[b1] / u[0, b1], 0.001) * al)
    cc2 = np.sqrt(np.maximum(c.gamma * p[b2] / u[0, b2], 0.001) * al)
    vn1 = np.abs((bw * u[1:4, b1]).sum(0) / u[0, b1])
    vn2 = np.abs((bw * u[1:4, b2]).sum(0) / u[0, b2])
    np.add.at(dt, b1, vn1 + (vn1 + vn2) + cc1 + (cc1 + cc2))
    np.add.at(dt, b2, vn2 + (vn1 + vn2) + cc2 + (cc1 + cc2))
    if c.ReynoldsNumber > 0:
        dv1 = 2.0 * np.maximum(am, mu[b1]) * al / u[0, b1]
        dv2 = 2.0 * np.maximum(am, mu[b2]) * al / u[0, b2]
        np.add.at(visc, b1, dv1 + (dv1 + dv2))
        np.add.at(visc, b2, dv2 + (dv1 + dv2))
    return 0.5 / (dt / g.V + visc / g.V ** 2)


def jst_scalar(c, g, u, p, dt):
    i1, i2 = g.i1, g.i2
    d = u[:, i1] - u[:, i2]
    d[4] = d[4] + p[i1] - p[i2]
    df = 1.0 / g.slen if c.useDissipationWeighting else np.ones(len(i1))
    lap = np.zeros((5, g.N))
    for k in range(5):
        np.add.at(lap[k], i1, -d[k] * df)
        np.add.at(lap[k], i2, d[k] * df)
    s7, s8 = np.zeros(g.N), np.zeros(g.N)
    np.add.at(s7, i1, -(p[i1] - p[i2]))
    np.add.at(s7, i2, p[i1] - p[i2])
    np.add.at(s8, i1, p[i1] + p[i2])
    np.add.at(s8, i2, p[i1] + p[i2])
    sens = 12.0 * np.abs(s7 / s8)
    lap = lap / g.conn
    d4v = lap[:, i1] - lap[:, i2]
    d2v = u[:, i1] - u[:, i2]
    d0 = np.minimum(g.V[i1] / dt[i1], g.V[i2] / dt[i2]) / (g.conn[i1] + g.conn[i2])
    d2 = d0 * c.secondOrderDissipationFactor * np.maximum(sens[i1], sens[i2])
    d4 = np.maximum(d0 * c.fourthOrderDissipationFactor - d2, 0.0)
    diss = np.zeros((5, g.N))
    for k in range(5):
        t = -d4v[k] * d4 + d2v[k] * d2
        np.add.at(diss[k], i1, t)
        np.add.at(diss[k], i2, -t)
    return diss


def viscous_term(c, g, u, p):
    """Returns (the term as added to the dissipation [5][N], mu, wall stress)."""
    i1, i2, b1, b2 = g.i1, g.i2, g.b1, g.b2
    gog = c.gamma / (c.gamma - 1.0)
    q = np.vstack([u[1:4] / u[0], gog * p / u[0]])  # u, v, w, T
    grad = np.zeros((3, 4, g.N))                     # d/dx_a of q_k
    for a in range(3):
        s = (q[:, i1] + q[:, i2]) * g.sw[a]
        sb = q[:, b1] + q[:, b2]
        for k in range(4):
            np.add.at(grad[a, k], i1, s[k])
            np.add.at(grad[a, k], i2, -s[k])
            np.add.at(grad[a, k], b1, (2.0 * q[k, b1] + sb[k]) * g.bw[a])
            np.add.at(grad[a, k], b2, (2.0 * q[k, b2] + sb[k]) * g.bw[a])
    grad = grad / g.V
    (dudx, dvdx, dwdx, dTdx), (dudy, dvdy, dwdy, dTdy), (dudz, dvdz, dwdz, dTdz) = grad
    T = np.maximum(gog * p / u[0], 0.001)
    T = np.where(T <= 0.001, 0.001, T)
    tc = (c.gamma - 1.0) * c.MachNumber ** 2
    tin = c.inflowTemperature
    mu = (1.0 / c.ReynoldsNumber) * ((tc * T) ** 1.5 * ((tin + 198.6) / (tc * tin * T + 198.6)))
    kk = mu / c.PrandtlNumber
    t = np.array([mu * (4.0 / 3.0 * dudx - 2.0 / 3.0 * (dvdy + dwdz)), mu * (dudy + dvdx), mu * (dudz + dwdx),
                  mu * (4.0 / 3.0 * dvdy - 2.0 / 3.0 * (dudx + dwdz)), mu * (dvdz + dwdy),
                  mu * (4.0 / 3.0 * dwdz - 2.0 / 3.0 * (dudx + dvdy)), kk * dTdx, kk * dTdy, kk * dTdz])
    # adiabatic wall on level 1: the normal temperature gradient removed
    n = g.normal[:, g.wall]
    dn = (t[6:9, g.wall] * n).sum(0)
    t[6:9, g.wall] = t[6:9, g.wall] - dn * n
    ws = np.zeros((3, g.N))
    nb = g.normal[:, g.bnodes]
    tb = t[:, g.bnodes]
    ws[0, g.bnodes] = tb[0] * nb[0] + tb[1] * nb[1] + tb[2] * nb[2]
    ws[1, g.bnodes] = tb[1] * nb[0] + tb[3] * nb[1] + tb[4] * nb[2]
    ws[2, g.bnodes] = tb[2] * nb[0] + tb[4] * nb[1] + tb[5] * nb[2]
    vel = u[1:4] / u[0]

    def flux(a, b, w):
        dt = t[:, a] + t[:, b]
        va, vb = vel[:, a], vel[:, b]
        dut = [va[0] * t[0, a] + vb[0] * t[0, b] + va[1] * t[1, a] + vb[1] * t[1, b] + va[2] * t[2, a]
               + vb[2] * t[2, b],
               va[0] * t[1, a] + vb[0] * t[1, b] + va[1] * t[3, a] + vb[1] * t[3, b] + va[2] * t[4, a]
               + vb[2] * t[4, b],
               va[0] * t[2, a] + vb[0] * t[2, b] + va[1] * t[4, a] + vb[1] * t[4, b] + va[2] * t[5, a]
               + vb[2] * t[5, b]]
        return np.array([w[0] * dt[0] + w[1] * dt[1] + w[2] * dt[2],
                         w[0] * dt[1] + w[1] * dt[3] + w[2] * dt[4],
                         w[0] * dt[2] + w[1] * dt[4] + w[2] * dt[5],
                         w[0] * (dt[6] + dut[0]) + w[1] * (dt[7] + dut[1]) + w[2] * (dt[8] + dut[2])])

    def own(a, w):
        va = vel[:, a]
        return 2.0 * np.array([w[0] * t[0, a] + w[1] * t[1, a] + w[2] * t[2, a],
                               w[0] * t[1, a] + w[1] * t[3, a] + w[2] * t[4, a],
                               w[0] * t[2, a] + w[1] * t[4, a] + w[2] * t[5, a],
                               w[0] * (t[6, a] + va[0] * t[0, a] + va[1] * t[1, a] + va[2] * t[2, a])
                               + w[1] * (t[7, a] + va[0] * t[1, a] + va[1] * t[3, a] + va[2] * t[4, a])
                               + w[2] * (t[8, a] + va[0] * t[2, a] + va[1] * t[4, a] + va[2] * t[5, a])])

    acc = np.zeros((4, g.N))
    f = flux(i1, i2, g.sw)
    for k in range(4):
        np.add.at(acc[k], i1, f[k])
        np.add.at(acc[k], i2, -f[k])
    keep = (g.bind != 2) & (g.bind != 9)
    a, b, w = g.b1[keep], g.b2[keep], g.bw[:, keep]
    f = flux(a, b, w)
    fa, fb = own(a, w), own(b, w)
    for k in range(4):
        np.add.at(acc[k], a, f[k] + fa[k])
        np.add.at(acc[k], b, f[k] + fb[k])
    term = np.zeros((5, g.N))
    term[1:] = -acc
    return term, mu, ws


def central_rhs(c, g, u, p):
    i1, i2 = g.i1, g.i2
    w = g.sw
    r, m, E = u[0], u[1:4], u[4]
    v = m / r
    rh = E + p
    rhs = np.zeros((5, g.N))
    f = np.zeros((5, len(i1)))
    f[0] = (w * (m[:, i1] + m[:, i2])).sum(0)
    for k in range(3):
        f[1 + k] = sum(w[a] * (m[k, i1] * v[a, i1] + m[k, i2] * v[a, i2]) for a in range(3)) \
            + w[k] * (p[i1] + p[i2])
    f[4] = (w * (rh[i1] * v[:, i1] + rh[i2] * v[:, i2])).sum(0)
    for k in range(5):
        np.add.at(rhs[k], i1, f[k])
        np.add.at(rhs[k], i2, -f[k])
    # boundary faces, boundaryTerm 1: node 1 gets |w|(3 F1 + F2), node 2 |w|(F1 + 3 F2)
    g1 = c.gamma - 1.0
    for b in range(len(g.b1)):
        a1, a2, ind = g.b1[b], g.b2[b], g.bind[b]
        wb = g.bw[:, b]
        rn = np.sqrt((wb ** 2).sum())
        if rn <= 1e-10:
            continue
        n = wb / rn

        def phys(i):
            vn = (v[:, i] * n).sum()
            return np.concatenate([[r[i] * vn], p[i] * n + r[i] * v[:, i] * vn, [rh[i] * vn]])

        def roe(i):
            inf = c.inflowField[6 * (ind - 3):6 * (ind - 3) + 6]
            ro, vo, eo, po = inf[0], np.array(inf[1:4]), inf[4], inf[5]
            epsr, hr = eo * ro, eo + po / ro
            unr = (vo * n).sum()
            fr = np.concatenate([[ro * unr], n * po + ro * vo * unr, [(epsr + po) * unr]])
            fl = phys(i)
            hl = rh[i] / r[i]
            di = np.sqrt(ro / r[i])
            d1 = 1.0 / (di + 1.0)
            vi = (di * vo + v[:, i]) * d1
            hi = (di * hr + hl) * d1
            ci2 = max(g1 * (hi - 0.5 * (vi ** 2).sum()), 1e-5)
            ci = np.sqrt(ci2)
            af = 0.5 * (vi ** 2).sum()
            ucp = (vi * n).sum()
            du = np.concatenate([[ro - r[i]], ro * vo - r[i] * v[:, i], [epsr - E[i]]])
            l1, l2, l3 = abs(ucp + ci), abs(ucp - ci), abs(ucp)
            s1, s2 = 0.5 * (l1 + l2), 0.5 * (l1 - l2)
            al1x = g1 * (af * du[0] - (vi * du[1:4]).sum() + du[4])
            al2x = -ucp * du[0] + (du[1:4] * n).sum()
            cc1 = (s1 - l3) * al1x / ci2 + s2 * al2x / ci
            cc2 = s2 * al1x / ci + (s1 - l3) * al2x
            diss = np.concatenate([[l3 * du[0] + cc1], l3 * du[1:4] + cc1 * vi + cc2 * n,
                                   [l3 * du[4] + cc1 * hi + cc2 * ucp]])
            return 0.5 * (fr + fl) - 0.5 * diss

        if ind <= 2 or ind == 9:
            F1, F2 = phys(a1), phys(a2)
        elif ind <= 4:
            F1, F2 = roe(a1), roe(a2)
        else:
            continue
        rhs[:, a1] += rn * (3.0 * F1 + F2)
        rhs[:, a2] += rn * (F1 + 3.0 * F2)
    return rhs


def _state(c, g, seed=9):
    u = initial_state(c, g.base, perturb_seed=seed, amplitude=0.05)
    k = np.arange(g.N)
    u[1] *= 1.0 + 0.03 * np.sin(k)
    u[2] = u[2] + 0.02 * np.cos(0.7 * k)
    u[3] = u[3] + 0.015 * np.sin(1.3 * k)
    u[4] *= 1.0 + 0.01 * np.cos(0.3 * k)
    return np.ascontiguousarray(u)


def _close(a, b):
    scale = np.abs(b).max(axis=-1, keepdims=True)
    scale = np.where(scale > 0, scale, 1.0)
    np.testing.assert_allclose(a / scale, b / scale, rtol=0, atol=TOL)


@pytest.fixture(scope="module")
def geo():
    return Geo(12, 4, 4)


@pytest.mark.parametrize("re,weighting", [(0.0, 0), (5000.0, 0), (0.0, 1)],
                         ids=["inviscid", "laminar", "dissipation_weighting"])
def test_time_steps_and_scalar_jst(geo, re, weighting):
    c = default_controls(ReynoldsNumber=re, fluxType=1, numberOfGridsToUse=1, wallsAreIsentropic=1,
                         secondOrderDissipationFactor=0.7, fourthOrderDissipationFactor=0.08,
                         useDissipationWeighting=weighting)
    o = Solver(c, geo.mesh, backend=oracle_backend())
    u = _state(c, geo)
    mu = np.zeros(geo.N)
    o.set_state(u)
    o.start()
    assert o.be.get_array(o._h, 1, b"mu", _ptr(mu)) == 0
    diss = np.zeros((5, geo.N))
    assert o.be.dissipation(o._h, 1, _ptr(u), _ptr(diss)) == 0
    dt_o = np.zeros(geo.N)
    assert o.be.get_array(o._h, 1, b"dt", _ptr(dt_o)) == 0
    p = np.abs(pressure(c, u))
    dt = time_steps(c, geo, u, p, mu)
    _close(dt, dt_o)
    ref = jst_scalar(c, geo, u, p, dt)
    assert np.all(np.abs(ref).max(axis=1) > 0)
    _close(diss, ref)


def test_viscous_term_sutherland_adiabatic_wall(geo):
    c = default_controls(ReynoldsNumber=5000.0, fluxType=1, numberOfGridsToUse=1, wallsAreIsentropic=1)
    o = Solver(c, geo.mesh, backend=oracle_backend())
    u = _state(c, geo, seed=4)
    d_o, mu_o, ws_o = np.zeros((5, geo.N)), np.zeros(geo.N), np.zeros((3, geo.N))
    assert o.be.viscous_term(o._h, 1, _ptr(u), _ptr(d_o), _ptr(mu_o), _ptr(ws_o)) == 0
    term, mu, ws = viscous_term(c, geo, u, np.abs(pressure(c, u)))
    _close(mu, mu_o)
    assert np.all(term[0] == 0) and np.all(d_o[0] == 0)
    _close(term[1:], d_o[1:])
    _close(ws, ws_o)


@pytest.mark.parametrize("alpha", [0.0, 4.0])
def test_central_residual_with_wall_and_far_field_faces(geo, alpha):
    c = default_controls(ReynoldsNumber=0.0, fluxType=1, numberOfGridsToUse=1, alpha=alpha, beta=1.5)
    o = Solver(c, geo.mesh, backend=oracle_backend())
    u = _state(c, geo, seed=6)
    assert {1, 2, 3} <= set(np.unique(geo.bind).tolist())
    _close(central_rhs(c, geo, u, pressure(c, u)), o.residual_fwd(u))


def _hops_from_boundary(g):
    far = np.full(g.N, 10 ** 6)
    far[g.bnodes] = 0
    adj = [[] for _ in range(g.N)]
    for a, b in zip(g.i1, g.i2):
        adj[a].append(b)
        adj[b].append(a)
    front = list(g.bnodes)
    d = 0
    while front:
        d += 1
        nxt = []
        for a in front:
            for b in adj[a]:
                if far[b] > d:
                    far[b] = d
                    nxt.append(b)
        front = nxt
    return far


@pytest.mark.parametrize("re", [0.0, 5000.0], ids=["inviscid", "laminar"])
def test_one_smoother_iteration_in_the_interior(re):
    g = Geo(16, 8, 8, seed=5)
    c = default_controls(ReynoldsNumber=re, fluxType=1, numberOfGridsToUse=1, CFLNumber=2.0,
                         wallsAreIsentropic=1, maxIncrementFactor=0.02)
    o = Solver(c, g.mesh, backend=oracle_backend())
    u0 = _state(c, g, seed=8)
    o.set_state(u0)
    o.start()
    u0 = o.get_state(1)  # start() applies the solution boundary conditions
    mu = np.zeros(g.N)
    assert o.be.get_array(o._h, 1, b"mu", _ptr(mu)) == 0
    o.do_time_iterations(1, 1, True, 1)
    got = o.get_state(1)

    p = np.abs(pressure(c, u0))
    dt = time_steps(c, g, u0, p, mu)
    diss = jst_scalar(c, g, u0, p, dt)
    if re > 0:
        diss = diss + viscous_term(c, g, u0, p)[0]
    u = u0.copy()
    for alpha in (0.6, 0.6, 1.0):
        rhs = central_rhs(c, g, u, pressure(c, u)) + diss
        delu = c.CFLNumber * alpha * (dt * rhs / g.V)
        new = u0 - delu
        big = np.abs(delu[0] / u0[0]) >= c.maxIncrementFactor
        new[0] = np.where(big, u0[0] - np.sign(delu[0]) * c.maxIncrementFactor * u0[0], new[0])
        new[0] = np.maximum(new[0], c.minimumDensity)
        u = new
    deep = _hops_from_boundary(g) >= 3
    assert deep.sum() > 50
    _close(u[:, deep], got[:, deep])
    assert np.abs(u[:, deep] - u0[:, deep]).max() > 1e-6


def viscous_term_compact(c, g, u, p):
    """makeViscosityTerm2 (def_par:5896-6807) from the Fortran: returns (the
    term as added to the dissipation [5][N], mu, wall stress)."""
    i1, i2, b1, b2 = g.i1, g.i2, g.b1, g.b2
    gog = c.gamma / (c.gamma - 1.0)
    q = np.vstack([u[1:4] / u[0], gog * p / u[0]])
    grad = np.zeros((3, 4, g.N))
    for a in range(3):
        s = (q[:, i1] + q[:, i2]) * g.sw[a]
        for k in range(4):
            np.add.at(grad[a, k], i1, s[k])
            np.add.at(grad[a, k], i2, -s[k])
            if c.boundaryTerm == 1:
                sb = q[:, b1] + q[:, b2]
                np.add.at(grad[a, k], b1, (2.0 * q[k, b1] + sb[k]) * g.bw[a])
                np.add.at(grad[a, k], b2, (2.0 * q[k, b2] + sb[k]) * g.bw[a])
            else:
                np.add.at(grad[a, k], b1, 4.0 * q[k, b1] * g.bw[a])
                np.add.at(grad[a, k], b2, 4.0 * q[k, b2] * g.bw[a])
    grad = grad / g.V
    T = np.maximum(gog * p / u[0], 0.001)
    tc = (c.gamma - 1.0) * c.MachNumber ** 2
    tin = c.inflowTemperature
    mu = (1.0 / c.ReynoldsNumber) * ((tc * T) ** 1.5 * ((tin + 198.6) / (tc * tin * T + 198.6)))
    kk = mu / c.PrandtlNumber
    G = grad.copy()                              # G[a, q] = scaled d q / d x_a
    G[:, :3] *= mu
    G[:, 3] *= kk
    n = g.normal[:, g.wall]
    dn = (G[:, 3, g.wall] * n).sum(0)
    G[:, 3, g.wall] -= dn * n

    def stress(Gn):
        # Gn[a, q] at some nodes -> (t1..t6)
        return np.array([4 / 3 * Gn[0, 0] - 2 / 3 * (Gn[1, 1] + Gn[2, 2]), Gn[1, 0] + Gn[0, 1],
                         Gn[2, 0] + Gn[0, 2], 4 / 3 * Gn[1, 1] - 2 / 3 * (Gn[0, 0] + Gn[2, 2]),
                         Gn[2, 1] + Gn[1, 2], 4 / 3 * Gn[2, 2] - 2 / 3 * (Gn[0, 0] + Gn[1, 1])])

    ws = np.zeros((3, g.N))
    t = stress(G[:, :, g.wall])
    ws[0, g.wall] = t[0] * n[0] + t[1] * n[1] + t[2] * n[2]
    ws[1, g.wall] = t[1] * n[0] + t[3] * n[1] + t[4] * n[2]
    ws[2, g.wall] = t[2] * n[0] + t[4] * n[1] + t[5] * n[2]
    if c.wallsAreIsentropic:
        G[:, 3, :g.Nb] = 0.0
    vel = np.vstack([u[1:4] * (1.0 / u[0]), gog * p * (1.0 / u[0])])
    inv = 1.0 / g.slen
    x = g.base.array(1, "coords")  # the coordinates the level descriptor carries
    r = (x[:, i2] - x[:, i1]) * inv
    S = G[:, :, i1] + G[:, :, i2]
    cf = np.array([mu[i1] + mu[i2]] * 3 + [kk[i1] + kk[i2]])
    for k in range(4):
        dr = (S[:, k] * r).sum(0)
        S[:, k] = S[:, k] - dr * r + cf[k] * (vel[k, i2] - vel[k, i1]) * inv * r
    dt = stress(S)
    av = 0.5 * (vel[:3, i1] + vel[:3, i2])
    dut = np.array([av[0] * dt[0] + av[1] * dt[1] + av[2] * dt[2], av[0] * dt[1] + av[1] * dt[3] + av[2] * dt[4],
                    av[0] * dt[2] + av[1] * dt[4] + av[2] * dt[5]])
    w = g.sw
    f = np.array([w[0] * dt[0] + w[1] * dt[1] + w[2] * dt[2], w[0] * dt[1] + w[1] * dt[3] + w[2] * dt[4],
                  w[0] * dt[2] + w[1] * dt[4] + w[2] * dt[5],
                  w[0] * (S[0, 3] + dut[0]) + w[1] * (S[1, 3] + dut[1]) + w[2] * (S[2, 3] + dut[2])])
    acc = np.zeros((4, g.N))
    for k in range(4):
        np.add.at(acc[k], i1, f[k])
        np.add.at(acc[k], i2, -f[k])
    keep = (g.bind != 2) & (g.bind != 9)
    for node, side in ((g.b1[keep], 0), (g.b2[keep], 1)):
        bw = g.bw[:, keep]
        tn = stress(G[:, :, node])
        tT = G[:, 3, node] * (0.0 if c.wallsAreIsentropic else 1.0)
        v = vel[:3, node]
        d = np.array([v[0] * tn[0] + v[1] * tn[1] + v[2] * tn[2], v[0] * tn[1] + v[1] * tn[3] + v[2] * tn[4],
                      v[0] * tn[2] + v[1] * tn[4] + v[2] * tn[5]])
        fb = 4.0 * np.array([bw[0] * tn[0] + bw[1] * tn[1] + bw[2] * tn[2],
                             bw[0] * tn[1] + bw[1] * tn[3] + bw[2] * tn[4],
                             bw[0] * tn[2] + bw[1] * tn[4] + bw[2] * tn[5],
                             bw[0] * (tT[0] + d[0]) + bw[1] * (tT[1] + d[1]) + bw[2] * (tT[2] + d[2])])
        for k in range(4):
            np.add.at(acc[k], node, fb[k])
    term = np.zeros((5, g.N))
    term[1:] = -acc
    return term, mu, ws


@pytest.mark.parametrize("isentropic,bterm", [(1, 1), (0, 1), (1, 2)], ids=["adiabatic", "isothermal", "fv_faces"])
def test_compact_viscous_term(geo, isentropic, bterm):
    # makeViscosityTerm2 (viscosityScheme 2): the compact stencil with the
    # edge-direction difference, on the jittered mesh's level 1
    c = default_controls(ReynoldsNumber=5000.0, fluxType=1, numberOfGridsToUse=1, wallsAreIsentropic=isentropic,
                         viscosityScheme=2, boundaryTerm=bterm)
    o = Solver(c, geo.mesh, backend=oracle_backend())
    u = _state(c, geo, seed=12)
    d_o, mu_o, ws_o = np.zeros((5, geo.N)), np.zeros(geo.N), np.zeros((3, geo.N))
    assert o.be.viscous_term(o._h, 1, _ptr(u), _ptr(d_o), _ptr(mu_o), _ptr(ws_o)) == 0
    term, mu, ws = viscous_term_compact(c, geo, u, np.abs(pressure(c, u)))
    _close(mu, mu_o)
    _close(term[1:], d_o[1:])
    _close(ws[:, geo.wall], ws_o[:, geo.wall])
    # the compact term differs from the wide one
    wide = viscous_term(default_controls(ReynoldsNumber=5000.0, wallsAreIsentropic=isentropic), geo, u,
                        np.abs(pressure(c, u)))[0]
    assert np.abs(wide[1:] - term[1:]).max() > 1e-6 * np.abs(term[1:]).max()


@pytest.mark.parametrize("re", [0.0, 5000.0], ids=["inviscid", "laminar"])
def test_one_explicit_iteration_in_the_interior(re):
    # explicit time stepping (explicit with flowType 1, def_par:386-394,
    # 1427-1442, 13598-13607): no time differences, and every node's solve
    # takes the smallest local time step of the level
    g = Geo(16, 8, 8, seed=5)
    c = default_controls(ReynoldsNumber=re, fluxType=1, numberOfGridsToUse=1, CFLNumber=1.0,
                         wallsAreIsentropic=1, maxIncrementFactor=0.02, flowType=1, physicalTimeStep=0.2,
                         explicit_=1)
    o = Solver(c, g.mesh, backend=oracle_backend())
    u0 = _state(c, g, seed=8)
    o.set_state(u0)
    o.start()
    u0 = o.get_state(1)
    mu = np.zeros(g.N)
    assert o.be.get_array(o._h, 1, b"mu", _ptr(mu)) == 0
    assert o.explicit_time_step() == 0.2  # the control's value until a time step is made
    o.do_time_iterations(1, 1, True, 1)
    got = o.get_state(1)

    p = np.abs(pressure(c, u0))
    dt = time_steps(c, g, u0, p, mu)
    dtg = dt.min()
    np.testing.assert_allclose(o.explicit_time_step(), dtg, rtol=TOL)
    diss = jst_scalar(c, g, u0, p, dt)
    if re > 0:
        diss = diss + viscous_term(c, g, u0, p)[0]
    u = u0.copy()
    for alpha in (0.6, 0.6, 1.0):
        rhs = central_rhs(c, g, u, pressure(c, u)) + diss
        delu = c.CFLNumber * alpha * (dtg * rhs / g.V)
        new = u0 - delu
        big = np.abs(delu[0] / u0[0]) >= c.maxIncrementFactor
        new[0] = np.where(big, u0[0] - np.sign(delu[0]) * c.maxIncrementFactor * u0[0], new[0])
        new[0] = np.maximum(new[0], c.minimumDensity)
        u = new
    deep = _hops_from_boundary(g) >= 3
    _close(u[:, deep], got[:, deep])
    assert np.abs(u[:, deep] - u0[:, deep]).max() > 1e-8
