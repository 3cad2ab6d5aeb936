"""Spalart-Allmaras (turbulenceModel 1) on the GPU against the CPU
restatement, bit for bit on every level (nu~ is the sixth state component).

The SA source term's exp and log are the pinned constructions shared by both
sides, so the states agree exactly; the residual norms (six with SA) are
reductions in another order and agree to 1e-12 relative.
"""
import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

pytestmark = pytest.mark.gpu

BASE = dict(ReynoldsNumber=1.0e5, MachNumber=0.5, CFLNumber=1.0, fluxType=1, numberOfGridsToUse=3,
            multigridScheme=3, turbulenceModel=1, wallsAreIsentropic=1)

CASES = {
    "sa_central": dict(),
    "sa_frozen_after_2": dict(numberOfTurbulenceSteps=2),
    "sa_turb_grids_3": dict(numberOfTurbulenceGrids=3, turbProlongationRelaxation=0.7),
    "sa_hllc2": dict(fluxType=4, HLLCFluxOrder=2, Automaticlipping=1),
    "sa_low_cap": dict(maxTurbulenceValue=0.2, turbulentCFLNumber=0.5),
    "sa_scheme1": dict(multigridScheme=1),
    "sa_scheme0": dict(multigridScheme=0),
    "sa_fv_boundary": dict(boundaryTerm=2),
    "sa_compact_viscous": dict(viscosityScheme=2),
}


def assert_same(g, o, what):
    for level in range(1, g.nlevels + 1):
        a, b = g.get_state(level), o.get_state(level)
        assert a.shape[0] == 6
        if not np.array_equal(a, b):
            d = np.abs(a - b)
            k, i = np.unravel_index(np.argmax(d), d.shape)
            raise AssertionError(f"{what}: level {level} differs, max {d.max():.3e} at comp {k} node {i}")


@pytest.mark.parametrize("name", list(CASES))
def test_sa_cycles_bitwise(name):
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    c = default_controls(**{**BASE, **CASES[name]})
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    u0 = initial_state(c, mesh, perturb_seed=20261203)
    for s in (g, o):
        s.set_state(u0)
        s.start()
    for cyc in range(1, 5):
        g.cycle(cyc)
        o.cycle(cyc)
        assert_same(g, o, f"{name} cycle {cyc}")
        rg, ro = g.residuals()[0], o.residuals()[0]
        assert rg.shape == (6,)
        np.testing.assert_allclose(rg, ro, rtol=1e-12, atol=0)


def test_sa_freestream_initialisation_and_eager_calls():
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=2)
    c = default_controls(**{**BASE, "numberOfGridsToUse": 2})
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    for s in (g, o):
        s.init_freestream()
        s.start()
    assert np.all(g.get_state(1)[5] == o.get_state(1)[5])
    # the solver steps one by one (outside the cycle graph), turbulence on/off
    for s in (g, o):
        s.do_time_iterations(1, 1, True, 1, calc_turb=True)
        s.restrict(1, calc_turb=False)
        s.do_time_iterations(2, 1, False, 1, calc_turb=False)
        s.prolong(2)
    assert_same(g, o, "eager steps")


def test_sa_rejected_without_viscosity():
    mesh = Mesh.bump_channel(6, 2, 2, 0.05, nlevels=1)
    c = default_controls(**{**BASE, "ReynoldsNumber": 0.0, "numberOfGridsToUse": 1})
    with pytest.raises(RuntimeError):
        Solver(c, mesh)


@pytest.mark.parametrize("flux", [1, 4])
def test_sa_naca0012_rans_bitwise(flux):
    # the RANS configuration's geometry (extruded NACA0012, M 0.8, alpha 1.25,
    # Re 6e6) at a coarse resolution: far field, airfoil wall and span
    # symmetry planes with the SA model
    mesh = Mesh.naca0012(64, 24, 4, first_cell=1e-3, growth=1.2, nlayer=10, farfield=10.0, span=0.5,
                         nlevels=3)
    c = default_controls(ReynoldsNumber=6.0e6, MachNumber=0.8, alpha=1.25, CFLNumber=1.0, fluxType=flux,
                         HLLCFluxOrder=2, Automaticlipping=1, multigridScheme=3, numberOfGridsToUse=3,
                         turbulenceModel=1, wallsAreIsentropic=1)
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    for s in (g, o):
        s.init_freestream()
        s.start()
    for cyc in range(1, 4):
        g.cycle(cyc)
        o.cycle(cyc)
        assert_same(g, o, f"naca flux {flux} cycle {cyc}")
    np.testing.assert_allclose(g.forces(), o.forces(), rtol=1e-12, atol=1e-15)
