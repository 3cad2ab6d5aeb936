"""CPU checks of the pieces of the steady adjoint that need no GPU.

* The oracle's dual-number tangent of one level-1 smoother iteration: its
  value part is the oracle's own iteration bit for bit, and its derivative
  part equals central differences of that iteration along random directions
  in the state and in the level-1 geometry (side_w, bnd_w, volume).
* The tangent of the lift and drag coefficients against central differences.
* fp_geometry rebuilds the level-1 arrays of a generated mesh bit for bit
  from its coordinates, and fp_geometry_vjp is the transpose of its
  derivative (dot product with central differences).
States carry random noise so that no |.|, min or max of the scheme sits on
its kink (the derivative is checked where it exists).
"""
import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

BASE = dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=2.0, numberOfGridsToUse=1)


def oracle_on(mesh, **ctl):
    c = default_controls(**{**BASE, **ctl})
    return c, Solver(c, mesh, backend=oracle_backend())


def generic_state(c, mesh, seed=7):
    u = initial_state(c, mesh, perturb_seed=3, amplitude=0.02)
    return np.ascontiguousarray(u + np.random.default_rng(seed).standard_normal(u.shape) * 0.01)


def iterate(c, mesh_like, u):
    s = Solver(c, mesh_like, backend=oracle_backend())
    s.set_state(u)
    s.do_time_iterations(1, 1, True, 1)
    return s.get_state(1)


@pytest.fixture(scope="module")
def mesh():
    return Mesh.bump_channel(12, 4, 4, 0.05, nlevels=1)


@pytest.mark.parametrize("ctl", [dict(), dict(boundaryTerm=0), dict(secondOrderDissipationFactor=0.0)])
def test_iteration_tangent(mesh, ctl):
    c, o = oracle_on(mesh, **ctl)
    u = generic_state(c, mesh)
    d = mesh.level(1)
    rng = np.random.default_rng(1)
    du = rng.standard_normal(u.shape)
    dsw = rng.standard_normal((3, d.n_sides)) * 1e-2
    dbw = rng.standard_normal((3, d.n_bsides)) * 1e-2
    dvol = rng.standard_normal(d.n_nodes) * 1e-3
    v, dv = o.iteration_jvp(u, du, dsw, dbw, dvol)
    assert np.array_equal(v, iterate(c, mesh, u))
    sw, bw, vol = mesh.array(1, "side_w"), mesh.array(1, "bnd_w"), mesh.array(1, "volume")
    h = 1e-6

    def G(t):
        m = mesh.with_level1_geometry(sw + t * dsw, bw + t * dbw, vol + t * dvol)
        return iterate(c, m, u + t * du)

    fd = (G(h) - G(-h)) / (2 * h)
    assert np.abs(fd - dv).max() <= 1e-8 * np.abs(dv).max()


@pytest.mark.parametrize("name", ["CL", "CD"])
def test_objective_tangent(mesh, name):
    c, o = oracle_on(mesh)
    u = generic_state(c, mesh)
    rng = np.random.default_rng(2)
    du = rng.standard_normal(u.shape)
    bw = mesh.array(1, "bnd_w")
    dbw = rng.standard_normal(bw.shape) * 1e-2
    J, dJ = o.objective_jvp(name, u, du, bnd_w=dbw)
    h = 1e-6

    def Jt(t):
        m = mesh.with_level1_geometry(mesh.array(1, "side_w"), bw + t * dbw, mesh.array(1, "volume"))
        s = Solver(c, m, backend=oracle_backend())
        return s.objective_jvp(name, u + t * du, np.zeros_like(u))[0]

    assert Jt(0.0) == J
    fd = (Jt(h) - Jt(-h)) / (2 * h)
    assert abs(fd - dJ) <= 1e-7 * abs(dJ)


def test_geometry_rebuilds_the_mesh_arrays():
    m = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=2)
    sw, bw, vol = m.geometry()
    assert np.array_equal(sw, m.array(1, "side_w"))
    assert np.array_equal(bw, m.array(1, "bnd_w"))
    assert np.array_equal(vol, m.array(1, "volume"))
    sw2, bw2, vol2 = m.geometry(m.array(1, "coords"))
    assert np.array_equal(sw2, sw) and np.array_equal(bw2, bw) and np.array_equal(vol2, vol)


def test_geometry_vjp_is_the_transpose():
    m = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=1)
    x = m.array(1, "coords")
    sw, bw, vol = m.geometry()
    rng = np.random.default_rng(0)
    dx = rng.standard_normal(x.shape)
    a, b, c = rng.standard_normal(sw.shape), rng.standard_normal(bw.shape), rng.standard_normal(vol.shape)
    xb = m.geometry_vjp(a, b, c)
    h = 1e-6
    p, q = m.geometry(x + h * dx), m.geometry(x - h * dx)
    fd = sum(((pp - qq) * w).sum() for pp, qq, w in zip(p, q, (a, b, c))) / (2 * h)
    assert abs(fd - (xb * dx).sum()) <= 1e-8 * abs(fd)


def test_geometry_needs_elements(tmp_path):
    m = Mesh.bump_channel(6, 2, 2, 0.05, nlevels=1)
    m.write_sol(tmp_path / "m.sol")
    r = Mesh.read_sol(tmp_path / "m.sol")
    with pytest.raises(RuntimeError):
        r.geometry()


LAMINAR = dict(ReynoldsNumber=500.0, CFLNumber=1.0)


@pytest.mark.parametrize("ctl", [dict(wallsAreIsentropic=1), dict(wallsAreIsentropic=0)])
def test_laminar_iteration_tangent(mesh, ctl):
    """The state of a laminar iteration is (u, mu): mu the viscosity the
    time step reads; the iteration also returns the viscosity of u."""
    c, o = oracle_on(mesh, **LAMINAR, **ctl)
    u = generic_state(c, mesh)
    n = u.shape[1]
    mu_u = o.iteration_jvp(u, np.zeros_like(u), mu=np.zeros(n), dmu=np.zeros(n))[2]
    # the value part is the oracle's own iteration with that viscosity read
    s = Solver(c, mesh, backend=oracle_backend())
    s.set_state(u)
    s.start()  # the wall condition on u and the viscosity 1/Re of the initial field
    us = s.get_state(1)
    v1, _, mu1, _ = o.iteration_jvp(us, np.zeros_like(u), mu=np.full(n, 1.0 / c.ReynoldsNumber), dmu=np.zeros(n))
    s.do_time_iterations(1, 1, True, 1)
    assert np.array_equal(v1, s.get_state(1))
    # the viscosity the iteration returns is that of its input state alone
    assert np.array_equal(o.iteration_jvp(us, np.zeros_like(u), mu=np.zeros(n), dmu=np.zeros(n))[2], mu1)
    mu = mu_u * (1 + 0.05 * np.random.default_rng(3).standard_normal(n))
    d = mesh.level(1)
    rng = np.random.default_rng(1)
    du = rng.standard_normal(u.shape)
    dmu = rng.standard_normal(n) * 1e-4
    dg = [rng.standard_normal((3, d.n_sides)) * 1e-2, rng.standard_normal((3, d.n_bsides)) * 1e-2,
          rng.standard_normal(n) * 1e-3]
    _, dv, _, dmo = o.iteration_jvp(u, du, *dg, mu=mu, dmu=dmu)
    base = [mesh.array(1, k) for k in ("side_w", "bnd_w", "volume")]
    h = 1e-6

    def G(t):
        m = mesh.with_level1_geometry(*[b + t * x for b, x in zip(base, dg)])
        return Solver(c, m, backend=oracle_backend()).iteration_jvp(u + t * du, np.zeros_like(u), mu=mu + t * dmu,
                                                                     dmu=np.zeros(n))
    a, b = G(h), G(-h)
    assert np.abs((a[0] - b[0]) / (2 * h) - dv).max() <= 1e-8 * np.abs(dv).max()
    assert np.abs((a[2] - b[2]) / (2 * h) - dmo).max() <= 1e-8 * np.abs(dmo).max()


@pytest.mark.parametrize("name", ["CL", "CD"])
def test_laminar_objective_tangent(mesh, name):
    c, o = oracle_on(mesh, **LAMINAR)
    u = generic_state(c, mesh)
    d = mesh.level(1)
    rng = np.random.default_rng(2)
    du = rng.standard_normal(u.shape)
    dg = [rng.standard_normal((3, d.n_sides)) * 1e-2, rng.standard_normal((3, d.n_bsides)) * 1e-2,
          rng.standard_normal(d.n_nodes) * 1e-3]
    J, dJ = o.objective_jvp(name, u, du, *dg)
    base = [mesh.array(1, k) for k in ("side_w", "bnd_w", "volume")]
    h = 1e-6

    def Jt(t):
        m = mesh.with_level1_geometry(*[b + t * x for b, x in zip(base, dg)])
        return Solver(c, m, backend=oracle_backend()).objective_jvp(name, u + t * du, np.zeros_like(u))[0]

    fd = (Jt(h) - Jt(-h)) / (2 * h)
    assert abs(fd - dJ) <= 1e-7 * abs(dJ)
