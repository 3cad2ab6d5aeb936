"""The GPU adjoint product (flite_residual_vjp) against the CPU tangent.

ubar = (dR/du)^T rbar must satisfy the dot-product identity
rbar . (J du) = ubar . du for the oracle's dual-number tangent J du, for any
rbar and du (tolerance 1e-11 relative to the magnitude of the terms), and the
central difference of the GPU residual itself along du (step 1e-5, tolerance
1e-6 relative).
"""
import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

pytestmark = pytest.mark.gpu

BASE = dict(ReynoldsNumber=0.0, fluxType=1, numberOfGridsToUse=3)


def pair(mesh, **ctl):
    c = default_controls(**{**BASE, **ctl})
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    u = initial_state(c, mesh, perturb_seed=13, amplitude=0.05)
    for s in (g, o):
        s.set_state(u)
        s.start()
    return c, g, o


@pytest.mark.parametrize("level", [1, 2, 3])
@pytest.mark.parametrize("boundary_term", [0, 1])
def test_vjp_dot_product_identity(level, boundary_term):
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    c, g, o = pair(mesh, boundaryTerm=boundary_term)
    u = o.get_state(level)
    rng = np.random.default_rng(100 + level)
    for _ in range(3):
        du = rng.standard_normal(u.shape)
        rbar = rng.standard_normal(u.shape)
        jv = o.residual_jvp(u, du, level=level)
        ub = g.residual_vjp(u, rbar, level=level)
        lhs, rhs = float(np.dot(rbar.ravel(), jv.ravel())), float(np.dot(ub.ravel(), du.ravel()))
        mag = float(np.abs(rbar * jv).sum())
        assert abs(lhs - rhs) <= 1e-11 * mag, (lhs, rhs, mag)


def test_vjp_against_central_difference_of_gpu_residual():
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    c, g, o = pair(mesh)
    u = g.get_state(1)
    rng = np.random.default_rng(3)
    du = rng.standard_normal(u.shape) * np.abs(u).max(axis=1, keepdims=True) * 1e-2
    rbar = rng.standard_normal(u.shape)
    h = 1e-5
    fd = (g.residual_fwd(u + h * du) - g.residual_fwd(u - h * du)) / (2 * h)
    ub = g.residual_vjp(u, rbar)
    lhs, rhs = float(np.dot(rbar.ravel(), fd.ravel())), float(np.dot(ub.ravel(), du.ravel()))
    assert abs(lhs - rhs) <= 1e-6 * float(np.abs(rbar * fd).sum())


def test_vjp_full_jacobian_on_a_small_level():
    # every row of J^T from the GPU equals the column of J from the tangent
    mesh = Mesh.bump_channel(6, 2, 2, 0.05, nlevels=1)
    c = default_controls(**{**BASE, "numberOfGridsToUse": 1})
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    u = initial_state(c, mesh, perturb_seed=2, amplitude=0.05)
    n = u.size
    J = np.zeros((n, n))
    for k in range(n):
        e = np.zeros(n)
        e[k] = 1.0
        J[:, k] = o.residual_jvp(u, e.reshape(u.shape)).ravel()
    JT = np.zeros((n, n))
    for k in range(n):
        e = np.zeros(n)
        e[k] = 1.0
        JT[:, k] = g.residual_vjp(u, e.reshape(u.shape)).ravel()
    np.testing.assert_allclose(JT, J.T, rtol=0, atol=1e-12 * np.abs(J).max())


def test_vjp_rejects_unsupported_flux():
    mesh = Mesh.bump_channel(6, 2, 2, 0.05, nlevels=1)
    c = default_controls(**{**BASE, "fluxType": 4, "numberOfGridsToUse": 1})
    g = Solver(c, mesh)
    u = initial_state(c, mesh)
    with pytest.raises(RuntimeError, match="status 2"):
        g.residual_vjp(u, u)


def test_adjoint_cost_ratio_is_measured():
    mesh = Mesh.bump_channel(48, 16, 16, 0.05, nlevels=1)
    c = default_controls(**{**BASE, "numberOfGridsToUse": 1})
    g = Solver(c, mesh)
    g.set_state(initial_state(c, mesh))
    fwd, vjp = g.profile_adjoint(level=1, reps=5)
    assert fwd > 0 and vjp > 0
