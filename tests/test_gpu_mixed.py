"""Mixed precision (FLITE_MIXED) against the FP64 CPU restatement.

FLITE_MIXED evaluates the interior central fluxes in FP32 as increments over
an FP64 anchor state (the state at the first stage of each relaxation step,
whose interior-edge residual is summed in FP64), and keeps FP64 for the
conserved-variable update, the boundary-edge (wall and far-field
characteristic) fluxes, the dissipation, the time steps and the residual
norms.  Its rounding error is relative to the increment, not to the flux, so
the iteration converges to the FP64 fixed point.  Stated error bounds:

* one residual evaluation at u1 anchored at u0: |r_mixed - r_fp64| <=
  1e-5 * max|r_fp64(u1) - r_fp64(u0)| per component, for a 5 % and for a
  1e-7 increment;
* state after 5 cycles: relative difference <= 1e-6;
* res1 reduced by 1e-8 within 1.2x the FP64 cycle count; lift and drag there
  within 1e-6 relative (or 1e-9 absolute for a coefficient near zero) of the
  FP64 result.
"""
import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

pytestmark = pytest.mark.gpu

BASE = dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=2.0, numberOfGridsToUse=3, multigridScheme=3)


def pair(mesh, **ctl):
    c64 = default_controls(**{**BASE, **ctl})
    c32 = default_controls(**{**BASE, **ctl, "precision": 1})
    return c64, Solver(c32, mesh), Solver(c64, mesh, backend=oracle_backend())


@pytest.mark.parametrize("size", [0.05, 1e-7])
def test_mixed_residual_error_is_relative_to_the_increment(size):
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    c, m, o = pair(mesh)
    u0 = initial_state(c, mesh, perturb_seed=9, amplitude=0.05)
    rng = np.random.default_rng(4)
    u1 = u0 * (1.0 + size * rng.uniform(-1.0, 1.0, u0.shape))
    m.set_state(u0)
    rm = m.residual_fwd(u1)
    ro1, ro0 = o.residual_fwd(u1), o.residual_fwd(u0)
    scale = np.abs(ro1 - ro0).max(axis=1, keepdims=True)
    assert np.all(np.abs(rm - ro1) <= 1e-5 * scale)


@pytest.mark.parametrize("ctl", [dict(), dict(ReynoldsNumber=5000.0, wallsAreIsentropic=1)])
def test_mixed_cycles_track_fp64(ctl):
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    c, m, o = pair(mesh, **ctl)
    u0 = initial_state(c, mesh, perturb_seed=20261203)
    for s in (m, o):
        s.set_state(u0)
        s.start()
    for cyc in range(1, 6):
        m.cycle(cyc)
        o.cycle(cyc)
    a, b = m.get_state(1), o.get_state(1)
    assert np.abs(a - b).max() <= 1e-6 * np.abs(b).max()


def test_mixed_converged_forces_within_1e6():
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=3)
    c64 = default_controls(**BASE)
    c32 = default_controls(**BASE, precision=1)
    out = []
    for c in (c64, c32):
        s = Solver(c, mesh)
        s.set_state(initial_state(c, mesh, perturb_seed=20261203))
        s.start()
        r0 = None
        for cyc in range(1, 3001):
            s.cycle(cyc)
            r = s.residuals()[0][0]
            r0 = r0 or r
            if r < 1e-8 * r0:
                break
        assert r < 1e-8 * r0, f"precision {c.precision} did not converge: {r / r0:.3e}"
        out.append((cyc, s.forces()))
    (n64, f64), (n32, f32) = out
    assert n32 <= 1.2 * n64, (n32, n64)
    for k in (0, 1):
        assert abs(f32[k] - f64[k]) <= max(1e-6 * abs(f64[k]), 1e-9), (k, f32[k], f64[k])


@pytest.mark.parametrize("lanes", [1, 8, 32])
def test_mixed_gather_lanes_agree(lanes):
    # the FP32 increment sums keep their order in every gather shape
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    c32 = default_controls(**BASE, precision=1)
    a, b = Solver(c32, mesh), Solver(c32, mesh)
    u0 = initial_state(c32, mesh, perturb_seed=20261203)
    for s in (a, b):
        s.set_state(u0)
        s.start()
    for level in (1, 2, 3):
        a.set_gather_lanes(level, 1)
        b.set_gather_lanes(level, lanes)
    for cyc in range(1, 4):
        a.cycle(cyc)
        b.cycle(cyc)
    assert np.array_equal(a.get_state(1), b.get_state(1))
