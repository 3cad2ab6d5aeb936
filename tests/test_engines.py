"""Engine boundary conditions on the CPU: the engine inlet sides of the
preprocessor (makeEngineInflowData, gen3d_boundary.f90:768-920, and their
agglomeration :1061-1099), their .sol records (def_par:852-864) single- and
multi-domain, and the conditions of the CPU restatement
(setBCsOnSolutionField def_par:4488-4918, setBCsOnIncrementField :5084-5125).

* the coefficients of each inlet's sides sum to half its outward area vector
  on every level (triangles and quadrilaterals);
* the records survive the .sol round trip and the multi-domain files;
* engineFlowType 1 scales the inlet momenta to the target mass flow, the
  exhausts hold the exhaust state ramped in over numberOfEORelaxationSteps
  cycles; engineFlowType 2 runs;
* moving meshes and the tangent products refuse engines.
"""
import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, host_controls, initial_state
from hybrid_meshes import box
from test_domains import assert_same_mesh

GAMMA, MACH = 1.4, 0.5


def rear_state(pressure_ratio=(1.05, 1.08), rho=(0.9, 0.95), ru=(0.5, 0.45), nu=(0.0, 0.0)):
    """enginesRearParameters(7,2): a consistent exhaust state per engine."""
    p0 = 1.0 / (GAMMA * MACH * MACH)
    out = []
    for e in range(2):
        p = pressure_ratio[e] * p0
        out += [rho[e], ru[e], 0.0, 0.0, p / (GAMMA - 1) + 0.5 * ru[e] ** 2 / rho[e], p, nu[e]]
    return out


def engine_controls(**kw):
    base = dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=1.5, numberOfGridsToUse=3, engineFlowType=1,
                enginesFrontMassFlow=[0.06, 0.05], enginesRearParameters=rear_state())
    return host_controls(**{**base, **kw})


def inlet_flows(mesh, u):
    """The mass flow sum of each inlet, sum (rho v)_1 . w + (rho v)_2 . w."""
    idx, w = mesh.array(1, "engine_idx"), mesh.array(1, "engine_w")
    out = []
    for e in (1, 2):
        sel = idx[2] == e
        a, b = idx[0][sel] - 1, idx[1][sel] - 1
        out.append(np.sum(np.einsum("ks,ks->s", u[1:4, a], w[:, sel]) +
                          np.einsum("ks,ks->s", u[1:4, b], w[:, sel])))
    return out


@pytest.mark.parametrize("kind", ["tet", "hex", "mixed"])
def test_inlet_sides_cover_half_the_inlet_area(kind):
    m = box(8, 4, 4, kind=kind, nlevels=3, engines=2)
    try:
        # outflow plane x = 3 + 0.2 y: the face area vector of one cell is
        # (d/dj x d/dk) = (0.0625, -0.0125, 0.00125); the inlets cover four
        # cells (a side on the line between the two takes the inlet number
        # of the face that registered it first)
        cell = np.array([0.0625, -0.0125, 0.00125])
        for level in (1, 2, 3):
            idx, w = m.array(level, "engine_idx"), m.array(level, "engine_w")
            assert set(idx[2]) == ({1, 2} if level == 1 else set(idx[2]) & {1, 2})
            assert np.all(idx[0] <= idx[1])
            np.testing.assert_allclose(w.sum(axis=1), 0.5 * 4 * cell, rtol=1e-12, atol=1e-15)
            # every inlet side joins two nodes of a boundary side of the level
            b = m.array(level, "bnd_idx")
            pairs = {(min(x, y), max(x, y)) for x, y in zip(b[0], b[1])}
            assert all((x, y) in pairs for x, y in zip(idx[0], idx[1]))
        # level 1 has no side twice; the engine nodes carry indicators 5..8
        idx = m.array(1, "engine_idx")
        assert len({(x, y) for x, y in zip(idx[0], idx[1])}) == idx.shape[1]
        reg = m.array(1, "node_reg")
        assert reg[-12 + 20] <= reg[-11 + 20] and reg[-8 + 20] <= reg[-7 + 20]
    finally:
        m.close()
    one = box(8, 4, 4, kind=kind, nlevels=2, engines=1)
    try:
        for level in (1, 2):
            idx, w = one.array(level, "engine_idx"), one.array(level, "engine_w")
            assert set(idx[2]) == {1}
            np.testing.assert_allclose(w.sum(axis=1), 0.5 * 4 * cell, rtol=1e-12, atol=1e-15)
    finally:
        one.close()


def test_sol_round_trip_keeps_the_engine_sides(tmp_path):
    m = box(8, 4, 4, kind="tet", nlevels=3, engines=2)
    try:
        m.write_sol(tmp_path / "e.sol")
        r = Mesh.read_sol(tmp_path / "e.sol")
        for level in (1, 2, 3):
            for name in ("engine_idx", "engine_w", "bnd_idx", "node_reg"):
                assert np.array_equal(m.array(level, name), r.array(level, name)), (level, name)
        r.close()
    finally:
        m.close()


@pytest.mark.parametrize("nd", [2, 3])
def test_engine_sides_in_the_domain_files(tmp_path, nd):
    m = box(8, 4, 4, kind="hex", nlevels=3, engines=2)
    try:
        m.write_sol_domains(tmp_path / "e", tmp_path / "plotreg.reg", nd)
        merged = Mesh.read_sol_domains(tmp_path / "e", tmp_path / "plotreg.reg")
        canon = m.canonical()
        assert_same_mesh(merged, canon)
        for level in (1, 2, 3):
            for name in ("engine_idx", "engine_w"):
                assert np.array_equal(merged.array(level, name), canon.array(level, name)), (level, name)
        merged.close()
        canon.close()
    finally:
        m.close()


@pytest.mark.parametrize("levels", [1, 3])
def test_mass_flow_type_1_meets_the_target(levels):
    # one engine: every inlet side joins two inlet nodes, so after the
    # conditions the inlet's mass flow is the target to round-off
    m = box(8, 4, 4, kind="tet", nlevels=3, engines=1)
    c = engine_controls(numberOfGridsToUse=levels)
    o = Solver(c, m, backend=oracle_backend())
    try:
        o.set_state(initial_state(c, m, perturb_seed=3, amplitude=0.01))
        o.start()
        for cyc in range(1, 6):
            o.cycle(cyc)
            u = o.get_state(1)
            assert np.all(np.isfinite(u))
            assert inlet_flows(m, u)[0] == pytest.approx(0.06, rel=1e-12)
    finally:
        o.close()
        m.close()


def test_exhausts_ramp_to_the_exhaust_state():
    m = box(8, 4, 4, kind="tet", nlevels=1, engines=2)
    steps = 4
    c = engine_controls(numberOfGridsToUse=1, numberOfEORelaxationSteps=steps)
    o = Solver(c, m, backend=oracle_backend())
    try:
        o.set_state(initial_state(c, m, perturb_seed=3, amplitude=0.01))
        o.start()
        reg, ind = m.array(1, "node_reg"), m.array(1, "node_ind")
        inflow = np.array(c.inflowField[:5])
        rear = np.array(c.enginesRearParameters).reshape(2, 7)
        for cyc in range(1, 7):
            o.cycle(cyc)
            u = o.get_state(1)
            rp = min((cyc - 1) / steps, 1.0)
            for e, r in ((0, -8), (1, -6)):
                nodes = ind[reg[r + 20] - 1:reg[r + 21]] - 1
                assert len(nodes) > 0
                want = (1.0 - rp) * inflow + rp * rear[e, :5]
                assert np.array_equal(u[:, nodes], np.repeat(want[:, None], len(nodes), axis=1)), (cyc, e)
    finally:
        o.close()
        m.close()


@pytest.mark.parametrize("ftype", [1, 2])
def test_engine_runs_converge_towards_a_steady_state(ftype):
    m = box(8, 4, 4, kind="hex", nlevels=3, engines=2)
    c = engine_controls(engineFlowType=ftype, engineBCRelaxation=0.8)
    o = Solver(c, m, backend=oracle_backend())
    try:
        o.set_state(initial_state(c, m, perturb_seed=5, amplitude=0.01))
        o.start()
        res = []
        for cyc in range(1, 41):
            o.cycle(cyc)
            res.append(o.residuals()[0][0])
        assert np.all(np.isfinite(res)) and np.all(np.isfinite(o.get_state(1)))
        assert min(res[-5:]) < res[0]
    finally:
        o.close()
        m.close()


def test_refusals():
    m = box(8, 4, 4, kind="tet", nlevels=1, engines=2)
    try:
        # engine sides of a moving mesh would change every step
        c = engine_controls(numberOfGridsToUse=1, flowType=2, physicalTimeStep=0.1)
        with pytest.raises(RuntimeError):
            Solver(c, m, backend=oracle_backend())
        x0 = m.array(1, "coords")
        with pytest.raises(RuntimeError):
            m.set_moving(x0, x0, x0, 2)
        # the tangent products are of the engine-free residual
        c = engine_controls(numberOfGridsToUse=1)
        o = Solver(c, m, backend=oracle_backend())
        o.set_state(initial_state(c, m))
        o.start()
        u = np.ascontiguousarray(o.get_state(1))
        with pytest.raises(RuntimeError):
            o.residual_jvp(u, u)
        o.close()
    finally:
        m.close()
