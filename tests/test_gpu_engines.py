"""Engine boundary conditions on the GPU against the CPU restatement, bit for
bit on every level after each cycle: engine faces' fluxes (def_par:
2447-2511), the increment conditions (:5084-5125), the exhaust states with
their ramp, and on level 1 the inlet mass flow (engineFlowType 1) or mass
flow function (2) with the no-inflow correction (:4488-4918), through every
pass that sets the conditions (RK stages, restrictGrid's fine step,
prolongateGrid, the start-up).  Meshes of tetrahedra and of hexahedra with
two engines whose inlets and exhausts touch; the central, Roe and HLLC
fluxes, both boundary terms, laminar walls, Spalart-Allmaras, a dual-time
run, and the node kernels with lanes per node.
"""
import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Solver, default_controls, initial_state
from hybrid_meshes import box
from test_engines import rear_state

pytestmark = pytest.mark.gpu

BASE = dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=1.5, numberOfGridsToUse=3, engineFlowType=1,
            enginesFrontMassFlow=[0.06, 0.05], enginesRearParameters=rear_state())

CASES = {
    "central": dict(),
    "central_ft2": dict(engineFlowType=2, enginesFrontMassFlow=[0.09, 0.07]),
    "ramp_relaxed": dict(numberOfEORelaxationSteps=4, engineBCRelaxation=0.7),
    "fv_boundary": dict(boundaryTerm=2),
    "roe": dict(fluxType=3, CFLNumber=1.0),
    "hllc2": dict(fluxType=4, HLLCFluxOrder=2, Automaticlipping=1, CFLNumber=1.0),
    "laminar": dict(ReynoldsNumber=500.0, wallsAreIsentropic=0, CFLNumber=1.0),
    "laminar_ft2": dict(ReynoldsNumber=500.0, wallsAreIsentropic=1, CFLNumber=1.0, engineFlowType=2,
                        enginesFrontMassFlow=[0.09, 0.07]),
    "sa": dict(ReynoldsNumber=1.0e5, turbulenceModel=1, wallsAreIsentropic=1, CFLNumber=1.0,
               enginesRearParameters=rear_state(nu=(0.2, 0.3)), numberOfEORelaxationSteps=3),
    "sa_ft2": dict(ReynoldsNumber=1.0e5, turbulenceModel=1, wallsAreIsentropic=1, CFLNumber=1.0, engineFlowType=2,
                   enginesFrontMassFlow=[0.09, 0.07], enginesRearParameters=rear_state(nu=(0.2, 0.3))),
    "dual_time": dict(flowType=1, physicalTimeStep=0.2, timeScheme=2),
    # a negative target turns the inlet's flow into the domain, which the
    # no-inflow correction turns back
    "inflow_corrected": dict(enginesFrontMassFlow=[-0.02, 0.05]),
}


def run_pair(c, mesh, cycles=4, lanes=0):
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    if lanes:
        for level in range(1, mesh.nlevels + 1):
            g.set_gather_lanes(level, lanes)
    u0 = initial_state(c, mesh, perturb_seed=11, amplitude=0.02)
    for s in (g, o):
        s.set_state(u0)
        s.start()
    return g, o


def assert_same(g, o, nlevels, what):
    for level in range(1, nlevels + 1):
        a, b = g.get_state(level), o.get_state(level)
        assert np.all(np.isfinite(b)), (what, level)
        assert np.array_equal(a, b), (what, level, np.abs(a - b).max())


@pytest.mark.parametrize("kind", ["tet", "hex"])
@pytest.mark.parametrize("name", list(CASES))
def test_engine_cycles_match(name, kind):
    mesh = box(8, 4, 4, kind=kind, nlevels=3, engines=2)
    c = default_controls(**{**BASE, **CASES[name]})
    g, o = run_pair(c, mesh)
    try:
        assert_same(g, o, 3, (name, "start"))
        for cyc in range(1, 5):
            if c.flowType == 1 and cyc == 3:
                for s in (g, o):
                    s.next_physical_step()
            g.cycle(cyc)
            o.cycle(cyc)
            assert_same(g, o, 3, (name, cyc))
            assert np.allclose(g.residuals()[0], o.residuals()[0], rtol=1e-12, atol=0)
            assert np.allclose(g.forces(), o.forces(), rtol=1e-12, atol=1e-300)
            # the pressure the conditions leave (the forces read it)
            assert np.array_equal(g.get_pressure(1), o.get_pressure(1)), (name, cyc)
    finally:
        g.close()
        o.close()
        mesh.close()


@pytest.mark.parametrize("lanes", [4, 16])
@pytest.mark.parametrize("ftype", [1, 2])
def test_engine_cycles_with_lanes_per_node(ftype, lanes):
    mesh = box(8, 4, 4, kind="tet", nlevels=3, engines=2)
    c = default_controls(**{**BASE, "engineFlowType": ftype, "enginesFrontMassFlow": [0.09, 0.07] if ftype == 2 else
                            [0.06, 0.05]})
    g, o = run_pair(c, mesh, lanes=lanes)
    try:
        for cyc in range(1, 4):
            g.cycle(cyc)
            o.cycle(cyc)
            assert_same(g, o, 3, (ftype, lanes, cyc))
    finally:
        g.close()
        o.close()
        mesh.close()


def test_engine_residual_matches():
    # makeRHS with engine faces alone (no node conditions involved)
    mesh = box(8, 4, 4, kind="hex", nlevels=1, engines=2)
    c = default_controls(**{**BASE, "numberOfGridsToUse": 1})
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    try:
        u = np.ascontiguousarray(initial_state(c, mesh, perturb_seed=4, amplitude=0.05))
        for s in (g, o):
            s.set_state(u)
            s.start()
        assert np.array_equal(g.residual_fwd(u), o.residual_fwd(u))
    finally:
        g.close()
        o.close()
        mesh.close()


def test_engine_refusals():
    import ctypes
    mesh = box(8, 4, 4, kind="tet", nlevels=1, engines=2)
    try:
        with pytest.raises(RuntimeError):
            Solver(default_controls(**{**BASE, "numberOfGridsToUse": 1, "flowType": 2, "physicalTimeStep": 0.1}),
                   mesh)
        s = Solver(default_controls(**{**BASE, "numberOfGridsToUse": 1}), mesh)
        s.set_state(initial_state(s.c, mesh))
        s.start()
        u = np.ascontiguousarray(s.get_state(1))
        r = np.zeros_like(u)
        assert s.be.residual_vjp(s._h, 1, u.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p),
                                 r.ctypes.data_as(ctypes.c_void_p)) == 2
        s.close()
    finally:
        mesh.close()


@pytest.mark.parametrize("ftype", [1, 2])
def test_engines_in_the_device_node_order(ftype):
    # the locality renumbering at the ABI maps the engine sides' nodes too
    from flite3d_b200.solver import set_node_order
    mesh = box(8, 4, 4, kind="tet", nlevels=3, engines=2)
    c = default_controls(**{**BASE, "engineFlowType": ftype,
                            "enginesFrontMassFlow": [0.09, 0.07] if ftype == 2 else [0.06, 0.05]})
    set_node_order(1)
    try:
        g = Solver(c, mesh)
    finally:
        set_node_order(0)
    o = Solver(c, mesh, backend=oracle_backend())
    try:
        u0 = initial_state(c, mesh, perturb_seed=11, amplitude=0.02)
        for s in (g, o):
            s.set_state(u0)
            s.start()
        for cyc in range(1, 4):
            g.cycle(cyc)
            o.cycle(cyc)
            assert_same(g, o, 3, (ftype, cyc))
    finally:
        g.close()
        o.close()
        mesh.close()


def test_engines_from_domain_files(tmp_path):
    # a parallel run's files with engine inlet sides, ingested, on the GPU
    from flite3d_b200 import Mesh
    mesh = box(8, 4, 4, kind="hex", nlevels=3, engines=2)
    mesh.write_sol_domains(tmp_path / "e", tmp_path / "plotreg.reg", 3)
    merged = Mesh.read_sol_domains(tmp_path / "e", tmp_path / "plotreg.reg")
    c = default_controls(**BASE)
    g, o = run_pair(c, merged)
    try:
        for cyc in range(1, 4):
            g.cycle(cyc)
            o.cycle(cyc)
            assert_same(g, o, 3, cyc)
    finally:
        g.close()
        o.close()
        merged.close()
        mesh.close()


def test_engine_cases_in_a_batch_keep_their_own_graphs():
    # the engine conditions have no case-group form: such cases run as their
    # own branches of the batch graph, each as its solve alone
    from flite3d_b200.solver import Batch
    mesh = box(8, 4, 4, kind="tet", nlevels=3, engines=2)
    cases = [(default_controls(**{**BASE, "alpha": a}), mesh) for a in (0.0, 2.0)]
    batch = Batch(cases)
    try:
        singles = [Solver(c, m) for c, m in cases]
        for (c, m), bs, ss in zip(cases, batch.cases, singles):
            u0 = initial_state(c, m, perturb_seed=5, amplitude=0.02)
            for s in (bs, ss):
                s.set_state(u0)
                s.start()
        for cyc in range(1, 3):
            batch.cycle(cyc)
            for s in singles:
                s.cycle(cyc)
        assert batch.groups() == 0
        for bs, ss in zip(batch.cases, singles):
            assert np.array_equal(bs.get_state(1), ss.get_state(1))
        for s in singles:
            s.close()
    finally:
        batch.close()
        mesh.close()


def test_engines_with_mixed_precision_run():
    # FLITE_MIXED takes the engine conditions in FP64 like every node step
    mesh = box(8, 4, 4, kind="tet", nlevels=3, engines=2)
    c = default_controls(**{**BASE, "precision": 1})
    s = Solver(c, mesh)
    try:
        s.set_state(initial_state(c, mesh, perturb_seed=11, amplitude=0.02))
        s.start()
        res = []
        for cyc in range(1, 11):
            s.cycle(cyc)
            res.append(s.residuals()[0][0])
        assert np.all(np.isfinite(s.get_state(1))) and res[-1] < res[0]
    finally:
        s.close()
        mesh.close()
