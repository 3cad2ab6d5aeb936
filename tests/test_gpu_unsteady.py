"""Unsteady dual time stepping (flowType 1 on a static mesh): the GPU library
against the CPU restatement, bit for bit on every level after each physical
time step, for the second-order backward difference (timeScheme 2) and the
first-order one, inviscid, laminar and with the Spalart-Allmaras model;
residual norms and forces to 1e-12.
"""
import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ctl", [dict(), dict(timeScheme=1), dict(ReynoldsNumber=500.0, CFLNumber=1.0),
                                 dict(multigridScheme=1, physicalTimeStep=0.05)])
def test_unsteady_steps_match(ctl):
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    base = dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=2.0, numberOfGridsToUse=3, flowType=1,
                physicalTimeStep=0.2)
    c = default_controls(**{**base, **ctl})
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    u0 = initial_state(c, mesh, perturb_seed=5, amplitude=0.05)
    for s in (g, o):
        s.set_state(u0)
        s.start()
    for step in range(1, 4):
        for it in range(1, 5):
            g.cycle(it)
            o.cycle(it)
        for level in range(1, 4):
            assert np.array_equal(g.get_state(level), o.get_state(level)), (step, level)
        rg, ro = g.residuals()[0], o.residuals()[0]
        assert np.allclose(rg, ro, rtol=1e-12, atol=0)
        assert np.allclose(g.forces(), o.forces(), rtol=1e-12, atol=1e-300)
        g.next_physical_step()
        o.next_physical_step()
    assert not np.array_equal(g.get_state(1), u0)


@pytest.mark.parametrize("ctl", [dict(), dict(numberOfTurbulenceSteps=2), dict(timeScheme=1)])
def test_unsteady_spalart_allmaras_steps_match(ctl):
    """Unsteady RANS: the time difference of nu~ comes before its convection,
    and alone when the turbulence is not recomputed."""
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    base = dict(ReynoldsNumber=1.0e5, MachNumber=0.5, CFLNumber=1.0, fluxType=1, numberOfGridsToUse=3,
                multigridScheme=3, turbulenceModel=1, wallsAreIsentropic=1, flowType=1, physicalTimeStep=0.2)
    c = default_controls(**{**base, **ctl})
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    u0 = initial_state(c, mesh, perturb_seed=20261203)
    for s in (g, o):
        s.set_state(u0)
        s.start()
    for step in range(1, 4):
        for it in range(1, 4):
            g.cycle(it)
            o.cycle(it)
        for level in range(1, 4):
            a, b = g.get_state(level), o.get_state(level)
            assert a.shape[0] == 6 and np.array_equal(a, b), (step, level)
        g.next_physical_step()
        o.next_physical_step()


@pytest.mark.parametrize("ctl", [dict(numberOfGridsToUse=1), dict(), dict(ReynoldsNumber=500.0, CFLNumber=0.5),
                                 dict(ReynoldsNumber=1.0e5, turbulenceModel=1, wallsAreIsentropic=1, CFLNumber=0.5)])
def test_explicit_time_stepping_matches(ctl):
    # explicit time stepping: no time differences, the smallest local time
    # step of the last makeTimeSteps for every node (on any level, the
    # reference's global ivd%physicalTimeStep), advancing the current time
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    base = dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=1.0, numberOfGridsToUse=3, flowType=1,
                physicalTimeStep=0.2, explicit_=1)
    c = default_controls(**{**base, **ctl})
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    u0 = initial_state(c, mesh, perturb_seed=5, amplitude=0.02)
    for s in (g, o):
        s.set_state(u0)
        s.start()
    t = 0.0
    for it in range(1, 7):
        g.cycle(it)
        o.cycle(it)
        dt = g.explicit_time_step()
        assert dt == o.explicit_time_step() and 0.0 < dt < 1.0
        t += dt
        for level in range(1, c.numberOfGridsToUse + 1):
            a, b = g.get_state(level), o.get_state(level)
            assert np.all(np.isfinite(b)), (it, level)
            assert np.array_equal(a, b), (it, level, np.abs(a - b).max())
        # the force sums run in another order on the device: a component
        # that cancels (the lateral force) is close to the scale of the others
        fg, fo = g.forces(), o.forces()
        np.testing.assert_allclose(fg, fo, rtol=1e-12, atol=1e-12 * np.abs(fo).max())
    assert t > 0.0
    g.close()
    o.close()
    mesh.close()
