"""GPU (CUDA sm_100a, FP64) against the CPU restatement of the reference.

The FP64 kernels evaluate every reference expression in the reference's
order without FMA contraction, and sum per-node contributions in the
reference's edge order, so states are compared bit for bit
(np.array_equal).  Only the reductions (residual L2 norms, forces) use a
different summation order on the GPU; they are compared to 1e-12 relative.
"""
import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, default_controls, initial_state

pytestmark = pytest.mark.gpu

RTOL_REDUCTION = 1e-12

BASE = dict(ReynoldsNumber=0.0, MachNumber=0.5, CFLNumber=2.0, numberOfGridsToUse=3,
            multigridScheme=3)

CASES = {
    "central_jst": dict(fluxType=1),
    "hllc2_autoclip": dict(fluxType=4, HLLCFluxOrder=2, Automaticlipping=1),
    "hllc2_noclip": dict(fluxType=4, HLLCFluxOrder=2, Automaticlipping=0, HLLCClipping=0.5),
    "hllc1": dict(fluxType=4, HLLCFluxOrder=1),
    "first_order_diss": dict(fluxType=1, dissipationScheme=3, coarseGridDissipationScheme=3),
    "fv_boundary_term": dict(fluxType=1, boundaryTerm=2),
    "alpha_beta": dict(fluxType=1, alpha=3.0, beta=2.0),
    "supersonic_hllc2": dict(fluxType=4, HLLCFluxOrder=2, Automaticlipping=1, MachNumber=1.3,
                             CFLNumber=1.0),
    "dissipation_weighting": dict(fluxType=1, useDissipationWeighting=1, CFLNumber=0.5,
                                  fourthOrderDissipationFactor=0.05),
    "relax_steps2": dict(fluxType=1, numberOfRelaxationSteps=2, prolongationRelaxation=0.8,
                         multigridBCRelaxation=0.5, maxIncrementFactor=0.05),
    "laminar_adiabatic": dict(fluxType=1, ReynoldsNumber=5000.0, wallsAreIsentropic=1),
    "laminar_isothermal": dict(fluxType=1, ReynoldsNumber=5000.0, wallsAreIsentropic=0,
                               CFLNumber=0.5),
    "laminar_hllc2": dict(fluxType=4, HLLCFluxOrder=2, Automaticlipping=1,
                          ReynoldsNumber=5000.0, wallsAreIsentropic=1),
    "matrix_dissipation": dict(fluxType=1, useMatrixDissipation=1),
    # dissipation scheme 1 (linearity preserving) on level 1: the Roe matrix
    # by default, the scalar coefficient under useMatrixDissipation
    "lp_dissipation": dict(fluxType=1, dissipationScheme=1, fourthOrderDissipationFactor=0.05),
    "lp_dissipation_scalar": dict(fluxType=1, dissipationScheme=1, useMatrixDissipation=1),
    "lp_dissipation_weighted": dict(fluxType=1, dissipationScheme=1, useDissipationWeighting=1,
                                    CFLNumber=0.5, fourthOrderDissipationFactor=0.05),
    "lp_dissipation_fv": dict(fluxType=1, dissipationScheme=1, boundaryTerm=2,
                              fourthOrderDissipationFactor=0.05),
    "laminar_lp_dissipation": dict(fluxType=1, dissipationScheme=1, ReynoldsNumber=5000.0,
                                   wallsAreIsentropic=1, fourthOrderDissipationFactor=0.05),
    "matrix_dissipation_harten": dict(fluxType=1, useMatrixDissipation=1, HartensCorrectionFactor=0.3,
                                      secondOrderDissipationFactor=0.6),
    "laminar_matrix_dissipation": dict(fluxType=1, useMatrixDissipation=1, ReynoldsNumber=5000.0,
                                       wallsAreIsentropic=1),
    # viscosityScheme 2 (makeViscosityTerm2, the compact stencil)
    "laminar_visc2_adiabatic": dict(fluxType=1, ReynoldsNumber=5000.0, wallsAreIsentropic=1, viscosityScheme=2),
    "laminar_visc2_isothermal": dict(fluxType=1, ReynoldsNumber=5000.0, wallsAreIsentropic=0, CFLNumber=0.5,
                                     viscosityScheme=2),
    "laminar_visc2_fv": dict(fluxType=1, ReynoldsNumber=5000.0, wallsAreIsentropic=1, viscosityScheme=2,
                             boundaryTerm=2),
    "laminar_visc2_hllc2": dict(fluxType=4, HLLCFluxOrder=2, Automaticlipping=1, ReynoldsNumber=5000.0,
                                wallsAreIsentropic=1, viscosityScheme=2),
    # forceCalcType 3 (calculateLiftAndDrag3): its face loads pass through
    # the reference's shared help array, which the cycles after it must not see
    "laminar_forces_type3": dict(fluxType=1, ReynoldsNumber=5000.0, wallsAreIsentropic=1, forceCalcType=3,
                                 alpha=2.0, beta=1.0),
    # the upwind MUSCL / Van Albada extension and the five-stage scheme (no
    # reference counterpart): the GPU against the same extension on the CPU
    "roe_muscl_va_rk5": dict(fluxType=3, reconstruction=1, rungeKuttaStages=5,
                             secondOrderDissipationFactor=0.0, fourthOrderDissipationFactor=0.0),
    "roe_muscl_va_jst": dict(fluxType=3, reconstruction=1),
    "central_rk5": dict(fluxType=1, rungeKuttaStages=5),
    "laminar_roe_muscl_va_rk5": dict(fluxType=3, reconstruction=1, rungeKuttaStages=5,
                                     secondOrderDissipationFactor=0.0,
                                     fourthOrderDissipationFactor=0.0, ReynoldsNumber=5000.0,
                                     wallsAreIsentropic=1),
}
SCHEMES = [0, 1, 2, 4, 5, 7]


def make_pair(mesh, **ctl):
    c = default_controls(**{**BASE, **ctl})
    g = Solver(c, mesh)
    o = Solver(c, mesh, backend=oracle_backend())
    u0 = initial_state(c, mesh, perturb_seed=20261203, amplitude=0.01)
    for s in (g, o):
        s.set_state(u0)
        s.start()
    return c, g, o


def assert_same_state(g, o, what=""):
    for level in range(1, g.nlevels + 1):
        a, b = g.get_state(level), o.get_state(level)
        if not np.array_equal(a, b):
            d = np.abs(a - b)
            k, i = np.unravel_index(np.argmax(d), d.shape)
            raise AssertionError(f"{what} level {level}: max |diff| {d.max():.3e} at comp {k} "
                                 f"node {i} ({a[k, i]!r} vs {b[k, i]!r})")


@pytest.fixture(scope="module")
def mesh():
    return Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)


@pytest.mark.parametrize("flux,extra", [
    (1, {}), (2, {}), (3, {}), (4, dict(HLLCFluxOrder=2, Automaticlipping=1)),
    (3, dict(reconstruction=1)),
])
def test_residual_bitwise(mesh, flux, extra):
    c, g, o = make_pair(mesh, fluxType=flux, **extra)
    u = initial_state(c, mesh, perturb_seed=7, amplitude=0.05)
    u[1] *= 1.0 + 0.02 * np.sin(np.arange(u.shape[1]))
    rg, ro = g.residual_fwd(u), o.residual_fwd(u)
    assert np.array_equal(rg, ro)
    # coarse levels run the same edge kernels
    for level in (2, 3):
        uc = g.get_state(level)
        assert np.array_equal(g.residual_fwd(uc, level), o.residual_fwd(uc, level))


@pytest.mark.parametrize("case", sorted(CASES))
def test_calls_and_cycles_bitwise(mesh, case):
    c, g, o = make_pair(mesh, **CASES[case])
    assert_same_state(g, o, "start")
    for s in (g, o):
        s.do_time_iterations(1, 1, True, 1)
    assert_same_state(g, o, "doTimeIterations")
    for s in (g, o):
        s.restrict(1)
    assert_same_state(g, o, "restrictGrid")
    for s in (g, o):
        s.do_time_iterations(2, 1, False, 1)
        s.prolong(2)
    assert_same_state(g, o, "prolongateGrid")
    for cyc in range(1, 4):
        for s in (g, o):
            s.cycle(cyc)
        assert_same_state(g, o, f"cycle {cyc}")
        rg, mg, ig = g.residuals()
        ro, mo, io = o.residuals()
        np.testing.assert_allclose(rg, ro, rtol=RTOL_REDUCTION)
        assert np.array_equal(mg, mo) and np.array_equal(ig, io)
        np.testing.assert_allclose(g.forces(), o.forces(), rtol=RTOL_REDUCTION, atol=1e-15)
    assert np.array_equal(g.get_pressure(1), o.get_pressure(1))


def test_least_squares_gradients_single_grid(mesh):
    c, g, o = make_pair(mesh, fluxType=4, HLLCFluxOrder=2, Automaticlipping=1, GradientMethod=2,
                        numberOfGridsToUse=1)
    for cyc in range(1, 4):
        for s in (g, o):
            s.cycle(cyc)
        assert_same_state(g, o, f"LS gradients cycle {cyc}")


@pytest.mark.parametrize("scheme", SCHEMES)
def test_multigrid_schemes_bitwise(mesh, scheme):
    c, g, o = make_pair(mesh, fluxType=1, multigridScheme=scheme)
    for cyc in range(1, 3):
        for s in (g, o):
            s.cycle(cyc)
        assert_same_state(g, o, f"scheme {scheme} cycle {cyc}")


def test_cycle_graph_replay_matches_eager(mesh):
    # flite_cycle replays a captured graph; do the same cycle call by call
    # through the individual entry points and compare
    c, g, o = make_pair(mesh, fluxType=1)
    c2, g2, _ = make_pair(mesh, fluxType=1)
    g.cycle(1)
    # growing V for 3 grids, spelled out (mg_par:1017-1058)
    g2.do_time_iterations(1, 1, True, 1)
    g2.restrict(1)
    g2.do_time_iterations(2, 1, False, 1)
    g2.restrict(2)
    g2.do_time_iterations(3, 1, False, 1)
    g2.prolong(3)
    g2.do_time_iterations(2, 1, True, 1)
    g2.restrict(2)
    g2.do_time_iterations(3, 1, False, 1)
    g2.prolong(3)
    g2.prolong(2)
    assert_same_state(g, g2, "graph vs eager")


def test_convergence_history_matches(mesh):
    # residual history of 30 cycles on a coarser mesh: the states stay
    # bitwise equal, the norms agree to the reduction tolerance
    m = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=3)
    c, g, o = make_pair(m, fluxType=1)
    for cyc in range(1, 31):
        g.cycle(cyc)
        o.cycle(cyc)
    assert_same_state(g, o, "30 cycles")
    np.testing.assert_allclose(g.residuals()[0], o.residuals()[0], rtol=RTOL_REDUCTION)


@pytest.mark.parametrize("opts", [(128, 128, 2), (64, 256, 1), (256, 64, 2)])
def test_launch_options_do_not_change_results(opts):
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    c, g, o = make_pair(mesh, fluxType=1, ReynoldsNumber=5000.0, wallsAreIsentropic=1)
    g.set_kernel_options(*opts)
    for cyc in range(1, 4):
        g.cycle(cyc)
        o.cycle(cyc)
    assert_same_state(g, o, f"options {opts}")


@pytest.mark.parametrize("lanes", [1, 4, 8, 16, 32])
@pytest.mark.parametrize("name", ["central_jst", "hllc2_autoclip", "laminar_adiabatic", "first_order_diss",
                                  "roe_muscl_va_rk5", "laminar_visc2_isothermal"])
def test_gather_lanes_match(name, lanes):
    # every gather shape (a thread, or a group of 4..32 lanes, per node) on
    # every level gives the reference's sums
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    c, g, o = make_pair(mesh, **CASES[name])
    for level in (1, 2, 3):
        g.set_gather_lanes(level, lanes)
    for cyc in range(1, 4):
        g.cycle(cyc)
        o.cycle(cyc)
    assert_same_state(g, o, f"{name} lanes {lanes}")


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("name", ["central_jst", "laminar_adiabatic", "fv_boundary_term", "dissipation_weighting",
                                  "matrix_dissipation"])
def test_tiled_gather_modes_match(name, mode, order):
    # the gathers of every level with a thread per node through the
    # incidence rows of 256-node blocks, staged in shared memory (modes 1, 2)
    # or not (3, 4), or through the incidence lists (0); in the caller's node
    # numbering and in the locality numbering
    from flite3d_b200.solver import set_node_order
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    try:
        set_node_order(order)
        c, g, o = make_pair(mesh, **CASES[name])
    finally:
        set_node_order(0)
    for level in (1, 2, 3):
        g.set_gather_lanes(level, 1)
        g.set_tiled_gather(level, mode)
    for cyc in range(1, 4):
        g.cycle(cyc)
        o.cycle(cyc)
    assert_same_state(g, o, f"{name} tiled mode {mode} order {order}")
    assert np.array_equal(g.residual_fwd(g.get_state(1)), o.residual_fwd(o.get_state(1)))


@pytest.mark.parametrize("fuse", [0, 1])
@pytest.mark.parametrize("name", ["central_jst", "laminar_adiabatic", "laminar_isothermal", "fv_boundary_term",
                                  "dissipation_weighting", "matrix_dissipation", "laminar_matrix_dissipation",
                                  "laminar_visc2_adiabatic", "first_order_diss", "relax_steps2"])
def test_gather_fusion_matches(name, fuse):
    # a thread per node on every level, the gathers that walk the same
    # incidence list sharing one walk (k_ts_lap, k_jflux_vgrad) or not
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    c, g, o = make_pair(mesh, **CASES[name])
    for level in (1, 2, 3):
        g.set_gather_lanes(level, 1)
        g.set_gather_fusion(level, fuse)
    for cyc in range(1, 4):
        g.cycle(cyc)
        o.cycle(cyc)
    assert_same_state(g, o, f"{name} fusion {fuse}")
    groups = g.profile_kernels(1, reps=1)
    assert set(groups) == set(Solver.KERNEL_GROUPS)


def test_node_order_changes_no_result():
    # the device's locality numbering against the caller's: the same states,
    # pressures, residual maxima and their (caller-numbered) nodes
    from flite3d_b200.solver import set_node_order
    mesh = Mesh.bump_channel(24, 8, 8, 0.05, nlevels=3)
    c = default_controls(**{**BASE, "ReynoldsNumber": 5000.0, "wallsAreIsentropic": 1, "fluxType": 1})
    u0 = initial_state(c, mesh, perturb_seed=20261203, amplitude=0.01)
    runs = []
    try:
        for order in (0, 1):
            set_node_order(order)
            s = Solver(c, mesh)
            s.set_state(u0)
            s.start()
            for cyc in range(1, 4):
                s.cycle(cyc)
            runs.append((s.get_state(1), s.get_state(2), s.get_state(3), s.get_pressure(1), s.residuals(),
                         s.forces(), s.residual_fwd(u0)))
    finally:
        set_node_order(0)
    a, b = runs
    for k in (0, 1, 2, 3, 6):
        assert np.array_equal(a[k], b[k]), k
    np.testing.assert_allclose(a[4][0], b[4][0], rtol=1e-12)
    assert np.array_equal(a[4][1], b[4][1]) and np.array_equal(a[4][2], b[4][2])
    np.testing.assert_allclose(a[5], b[5], rtol=1e-12, atol=1e-15)
