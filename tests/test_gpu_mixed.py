"""Mixed precision (FLITE_MIXED) against the FP64 CPU restatement.

FLITE_MIXED computes the interior edge fluxes in FP32 from FP32 shadows of
the state into an FP32 edge buffer, sums them per node with compensated
(TwoSum) FP32 accumulation, and keeps FP64 for the conserved-variable update,
the boundary-edge (wall and far-field characteristic) fluxes, the dissipation,
the time steps and the residual norms.  Stated error bounds against FP64:

* one residual evaluation: |r_mixed - r_fp64| <= 2e-5 * max|r| per component;
* state after 5 cycles: relative difference <= 1e-6;
* converged (res1 reduced 1e-8) lift and drag: within 1e-6 relative (or 1e-9
  absolute for a coefficient near zero) of the FP64 result.
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


def test_mixed_residual_error_bound():
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    c, m, o = pair(mesh)
    u = initial_state(c, mesh, perturb_seed=9, amplitude=0.05)
    rm, ro = m.residual_fwd(u), o.residual_fwd(u)
    scale = np.abs(ro).max(axis=1, keepdims=True)
    assert np.all(np.abs(rm - ro) <= 2e-5 * scale)


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
    for k in (0, 1):
        assert abs(f32[k] - f64[k]) <= max(1e-6 * abs(f64[k]), 1e-9), (k, f32[k], f64[k])
