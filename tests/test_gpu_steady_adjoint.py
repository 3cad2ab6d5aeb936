"""The GPU steady adjoint (flite_iteration_vjp, flite_adjoint_solve).

* flite_iteration_vjp is the transpose of the oracle's dual-number tangent of
  one level-1 smoother iteration: lam . (G_u du + G_g dg) equals
  ubar . du + gbar . dg for random lam, du and geometry directions dg, at a
  generic state and at a converged one (1e-11 relative to the terms).
* flite_adjoint_solve (GMRES, and the fixed-point iteration, which agree):
  dCL/dX and dCD/dX (through fp_geometry_vjp) along
  the normal displacement of seeded wall nodes against the oracle's FP64
  tangent solve (the forward sensitivity of the same fixed point, 1e-7) and
  against central differences of converged GPU solutions on moved meshes
  (step 1e-6 of the channel height, 1e-5).  The meshes have jittered
  interior nodes, so no two edges tie in the dissipation's min/max switches.
* The same for laminar runs, whose iteration state also holds the viscosity
  the time step reads.
* The adjoint leaves the solution as it was, and refuses controls it does
  not cover.
"""
import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

pytestmark = pytest.mark.gpu

BASE = dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=2.0, multigridScheme=3)


def controls(**ctl):
    return default_controls(**{**BASE, **ctl})


class Jittered:
    """A generated bump channel whose level-1 interior nodes are moved by a
    seeded random fraction of the spacing (boundary nodes stay)."""

    def __init__(self, nx, ny, nz, nlevels, seed=11, frac=0.15):
        self.base = Mesh.bump_channel(nx, ny, nz, 0.05, nlevels=nlevels)
        x = self.base.array(1, "coords")
        jit = np.random.default_rng(seed).uniform(-1, 1, x.shape) * frac / nz
        jit[:, :self.base.level(1).n_bnodes] = 0.0
        self.X = x + jit
        self.mesh = self.at(self.X)

    def at(self, X):
        return self.base.with_level1_geometry(*self.base.geometry(X))

    def coords_sensitivity(self, r):
        return self.base.geometry_vjp(r["side_w_bar"], r["bnd_w_bar"], r["volume_bar"], xyz=self.X)

    def wall_nodes_and_normals(self):
        reg, ind = self.base.array(1, "node_reg"), self.base.array(1, "node_ind")
        wall = ind[reg[0] - 1:reg[1]] - 1
        bw, bidx = self.base.array(1, "bnd_w"), self.base.array(1, "bnd_idx")
        a = np.zeros_like(self.X)
        for k in range(2):
            np.add.at(a, (slice(None), bidx[k] - 1), -bw)
        return wall, a / np.linalg.norm(a, axis=0).clip(1e-300)


def converge(c, mesh, u0=None, tol=1e-14, max_cycles=4000):
    s = Solver(c, mesh)
    s.set_state(initial_state(c, mesh) if u0 is None else u0)
    s.start()
    res = None
    for it in range(1, max_cycles + 1):
        s.cycle(it)
        if it % 50 == 0:
            res = s.residuals()[0][0]
            if res < tol:
                break
    return s, res


def dot_check(g, o, u, seed):
    d = g.mesh.level(1)
    rng = np.random.default_rng(seed)
    du = rng.standard_normal(u.shape)
    dg = [rng.standard_normal((3, d.n_sides)) * 1e-2, rng.standard_normal((3, d.n_bsides)) * 1e-2,
          rng.standard_normal(d.n_nodes) * 1e-3]
    lam = rng.standard_normal(u.shape)
    _, dv = o.iteration_jvp(u, du, *dg)
    ub, *gb = g.iteration_vjp(u, lam, geometry=True)
    lhs = (lam * dv).sum()
    terms = [(ub * du).sum()] + [(a * b).sum() for a, b in zip(gb, dg)]
    scale = sum(abs(t) for t in terms) + abs(lhs)
    assert abs(lhs - sum(terms)) <= 1e-11 * scale, (lhs, terms)


@pytest.mark.parametrize("ctl", [dict(), dict(boundaryTerm=0), dict(secondOrderDissipationFactor=0.0),
                                 dict(fourthOrderDissipationFactor=0.0, CFLNumber=1.5)])
def test_iteration_vjp_is_the_transpose_of_the_tangent(ctl):
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=1)
    c = controls(numberOfGridsToUse=1, **ctl)
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    u = initial_state(c, mesh, perturb_seed=3, amplitude=0.02)
    u = u + np.random.default_rng(7).standard_normal(u.shape) * 0.01
    for s in (g, o):
        s.set_state(u)
        s.start()
    for seed in (1, 2):
        dot_check(g, o, u, seed)


def test_iteration_vjp_at_a_converged_state():
    j = Jittered(12, 4, 4, nlevels=2)
    c = controls(numberOfGridsToUse=2)
    s, res = converge(c, j.mesh)
    assert res < 1e-13
    u = s.get_state(1)
    c1 = controls(numberOfGridsToUse=1)
    g, o = Solver(c1, j.mesh), Solver(c1, j.mesh, backend=oracle_backend())
    for x in (g, o):
        x.set_state(u)
        x.start()
    dot_check(g, o, u, 3)


@pytest.fixture(scope="module")
def small_case():
    j = Jittered(16, 6, 6, nlevels=2)
    c = controls(numberOfGridsToUse=2)
    s, res = converge(c, j.mesh)
    return j, c, s, res


@pytest.mark.parametrize("name", ["CL", "CD"])
def test_adjoint_matches_the_cpu_tangent(small_case, name):
    j, c, s, res = small_case
    assert res < 1e-13
    u = s.get_state(1)
    r = s.adjoint_solve(name, tol=1e-13, max_iter=200000)
    assert r["residual"] <= 1e-13
    assert np.array_equal(s.get_state(1), u)  # the solution is left as it was
    assert r["J"] == s.objective(name)
    xb = j.coords_sensitivity(r)
    wall, nrm = j.wall_nodes_and_normals()
    o = Solver(controls(numberOfGridsToUse=1), j.mesh, backend=oracle_backend())
    for k in np.random.default_rng(21).choice(wall, 2, replace=False):
        dX = np.zeros_like(j.X)
        dX[:, k] = nrm[:, k]
        h = 1e-6
        gp, gm = j.base.geometry(j.X + h * dX), j.base.geometry(j.X - h * dX)
        dg = [(a - b) / (2 * h) for a, b in zip(gp, gm)]
        du = np.zeros_like(u)
        for _ in range(40000):
            _, dv = o.iteration_jvp(u, du, *dg)
            done = np.abs(dv - du).max() <= 1e-14 * max(1.0, np.abs(dv).max())
            du = dv
            if done:
                break
        _, dJ = o.objective_jvp(name, u, du, *dg)
        adj = (xb[:, k] * nrm[:, k]).sum()
        assert abs(adj - dJ) <= 1e-7 * abs(dJ), (k, adj, dJ)


def test_adjoint_matches_central_differences():
    j = Jittered(24, 8, 8, nlevels=3)
    c = controls(numberOfGridsToUse=3)
    s, res = converge(c, j.mesh)
    assert res < 1e-14
    u = s.get_state(1)
    r = s.adjoint_solve("CL", tol=1e-12, max_iter=200000)
    xb = j.coords_sensitivity(r)
    wall, nrm = j.wall_nodes_and_normals()
    h = 1e-6
    for k in np.random.default_rng(4).choice(wall, 4, replace=False):
        dX = np.zeros_like(j.X)
        dX[:, k] = nrm[:, k] * h
        Jp = converge(c, j.at(j.X + dX), u0=u, tol=1e-15, max_cycles=2000)[0].objective("CL")
        Jm = converge(c, j.at(j.X - dX), u0=u, tol=1e-15, max_cycles=2000)[0].objective("CL")
        fd = (Jp - Jm) / (2 * h)
        adj = (xb[:, k] * nrm[:, k]).sum()
        assert abs(adj - fd) <= 1e-5 * abs(fd), (k, adj, fd)


def test_gmres_and_fixed_point_agree(small_case):
    j, c, s, res = small_case
    r1 = s.adjoint_solve("CL", tol=1e-12, max_iter=200000)
    s.set_adjoint_method("fixed-point")
    r2 = s.adjoint_solve("CL", tol=1e-12, max_iter=200000)
    s.set_adjoint_method("gmres")
    assert r1["residual"] <= 1e-12 and r2["residual"] <= 1e-12
    assert r1["iterations"] < r2["iterations"]
    for k in ("side_w_bar", "bnd_w_bar"):
        assert np.abs(r1[k] - r2[k]).max() <= 1e-9 * np.abs(r2[k]).max()


def test_adjoint_leaves_the_solve_unchanged():
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=2)
    c = controls(numberOfGridsToUse=2)
    a, _ = converge(c, mesh, max_cycles=100, tol=0.0)
    b, _ = converge(c, mesh, max_cycles=100, tol=0.0)
    a.adjoint_solve("CD", tol=1e-6, max_iter=50)
    for it in range(101, 111):
        a.cycle(it)
        b.cycle(it)
    assert np.array_equal(a.get_state(1), b.get_state(1))


@pytest.mark.parametrize("ctl", [dict(ReynoldsNumber=5e6, turbulenceModel=1), dict(fluxType=4),
                                 dict(dissipationScheme=3), dict(flowType=1, physicalTimeStep=0.1),
                                 dict(rungeKuttaStages=5), dict(useMatrixDissipation=1),
                                 dict(dissipationScheme=1)])
def test_adjoint_refuses_what_it_does_not_cover(ctl):
    mesh = Mesh.bump_channel(6, 2, 2, 0.05, nlevels=1)
    c = controls(numberOfGridsToUse=1, **ctl)
    s = Solver(c, mesh)
    s.set_state(initial_state(c, mesh))
    s.start()
    with pytest.raises(RuntimeError, match="status 2"):
        s.adjoint_solve("CL")
    with pytest.raises(RuntimeError, match="status 2"):
        s.objective("CL")


# ---- laminar runs: the iteration's state is (u, mu), mu the viscosity the
# time step reads (makeTimeSteps runs before makeViscosityTerm)

LAMINAR = dict(ReynoldsNumber=500.0, CFLNumber=1.0, wallsAreIsentropic=1)


def viscosity_of(o, u):
    """mu of the state u: the viscosity makeViscosityTerm computes (oracle)."""
    n = u.shape[1]
    return o.iteration_jvp(u, np.zeros_like(u), mu=np.zeros(n), dmu=np.zeros(n))[2]


def laminar_dot_check(g, o, u, mu, seed):
    d = g.mesh.level(1)
    rng = np.random.default_rng(seed)
    du = rng.standard_normal(u.shape)
    dmu = rng.standard_normal(mu.shape) * 1e-3
    dg = [rng.standard_normal((3, d.n_sides)) * 1e-2, rng.standard_normal((3, d.n_bsides)) * 1e-2,
          rng.standard_normal(d.n_nodes) * 1e-3]
    lam = rng.standard_normal(u.shape)
    lam_mu = rng.standard_normal(mu.shape) * 1e2
    _, dv, _, dmo = o.iteration_jvp(u, du, *dg, mu=mu, dmu=dmu)
    ub, *gb, mub = g.iteration_vjp(u, lam, geometry=True, mu=mu, lam_mu=lam_mu)
    lhs = (lam * dv).sum() + (lam_mu * dmo).sum()
    terms = [(ub * du).sum(), (mub * dmu).sum()] + [(a * b).sum() for a, b in zip(gb, dg)]
    scale = sum(abs(t) for t in terms) + abs(lhs)
    assert abs(lhs - sum(terms)) <= 1e-11 * scale, (lhs, terms)


@pytest.mark.parametrize("ctl", [dict(), dict(wallsAreIsentropic=0), dict(boundaryTerm=0)])
def test_laminar_iteration_vjp_is_the_transpose_of_the_tangent(ctl):
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=1)
    c = controls(numberOfGridsToUse=1, **{**LAMINAR, **ctl})
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    u = initial_state(c, mesh, perturb_seed=3, amplitude=0.02)
    u = u + np.random.default_rng(7).standard_normal(u.shape) * 0.01
    for s in (g, o):
        s.set_state(u)
        s.start()
    # viscosities on both sides of the 1/Re floor of the time step
    mu = viscosity_of(o, u) * (1 + 0.05 * np.random.default_rng(3).standard_normal(u.shape[1]))
    for seed in (1, 2):
        laminar_dot_check(g, o, u, mu, seed)


@pytest.fixture(scope="module")
def laminar_case():
    j = Jittered(16, 6, 6, nlevels=2)
    c = controls(numberOfGridsToUse=2, **LAMINAR)
    s, res = converge(c, j.mesh, tol=1e-14, max_cycles=8000)
    return j, c, s, res


@pytest.mark.parametrize("name", ["CL", "CD"])
def test_laminar_adjoint_matches_the_cpu_tangent(laminar_case, name):
    j, c, s, res = laminar_case
    assert res < 1e-13
    u = s.get_state(1)
    r = s.adjoint_solve(name, tol=1e-13, max_iter=200000)
    assert r["residual"] <= 1e-13
    assert np.array_equal(s.get_state(1), u)
    assert r["J"] == s.objective(name)
    xb = j.coords_sensitivity(r)
    wall, nrm = j.wall_nodes_and_normals()
    o = Solver(controls(numberOfGridsToUse=1, **LAMINAR), j.mesh, backend=oracle_backend())
    mu = viscosity_of(o, u)
    J0, _ = o.objective_jvp(name, u, np.zeros_like(u))
    assert abs(J0 - r["J"]) <= 1e-12 * abs(J0)
    for k in np.random.default_rng(21).choice(wall, 2, replace=False):
        dX = np.zeros_like(j.X)
        dX[:, k] = nrm[:, k]
        h = 1e-6
        gp, gm = j.base.geometry(j.X + h * dX), j.base.geometry(j.X - h * dX)
        dg = [(a - b) / (2 * h) for a, b in zip(gp, gm)]
        du, dmu = np.zeros_like(u), np.zeros_like(mu)
        for _ in range(60000):
            _, dv, _, dmv = o.iteration_jvp(u, du, *dg, mu=mu, dmu=dmu)
            done = max(np.abs(dv - du).max(), np.abs(dmv - dmu).max() * 1e3) <= 1e-14 * max(1.0, np.abs(dv).max())
            du, dmu = dv, dmv
            if done:
                break
        _, dJ = o.objective_jvp(name, u, du, *dg)
        adj = (xb[:, k] * nrm[:, k]).sum()
        assert abs(adj - dJ) <= 1e-7 * abs(dJ), (k, adj, dJ)


def test_laminar_adjoint_matches_central_differences(laminar_case):
    j, c, s, res = laminar_case
    u = s.get_state(1)
    r = s.adjoint_solve("CD", tol=1e-12, max_iter=200000)
    xb = j.coords_sensitivity(r)
    wall, nrm = j.wall_nodes_and_normals()
    h = 1e-6
    for k in np.random.default_rng(6).choice(wall, 3, replace=False):
        dX = np.zeros_like(j.X)
        dX[:, k] = nrm[:, k] * h
        Jp = converge(c, j.at(j.X + dX), u0=u, tol=1e-15, max_cycles=3000)[0].objective("CD")
        Jm = converge(c, j.at(j.X - dX), u0=u, tol=1e-15, max_cycles=3000)[0].objective("CD")
        fd = (Jp - Jm) / (2 * h)
        adj = (xb[:, k] * nrm[:, k]).sum()
        assert abs(adj - fd) <= 1e-5 * abs(fd), (k, adj, fd)


@pytest.mark.parametrize("lam", [dict(), LAMINAR])
def test_mixed_precision_solution_has_the_fp64_sensitivities(lam):
    """FLITE_MIXED converges to the FP64 iteration's fixed point, so the
    adjoint of its solution (computed in FP64) equals the FP64 run's."""
    j = Jittered(12, 4, 4, nlevels=2)
    out = []
    for prec in (0, 1):
        c = controls(numberOfGridsToUse=2, precision=prec, **lam)
        s, res = converge(c, j.mesh, tol=1e-14, max_cycles=8000)
        assert res < 1e-13
        r = s.adjoint_solve("CL", tol=1e-12, max_iter=200000)
        out.append((s.get_state(1), r))
    (u0, r0), (u1, r1) = out
    assert np.abs(u1 - u0).max() <= 1e-11 * np.abs(u0).max()
    assert abs(r1["J"] - r0["J"]) <= 1e-10 * abs(r0["J"])
    for k in ("side_w_bar", "bnd_w_bar"):
        assert np.abs(r1[k] - r0[k]).max() <= 1e-8 * np.abs(r0[k]).max()
