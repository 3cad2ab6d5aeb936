"""Moving meshes (flowType 2) on the CPU: the geometry of a physical step
(gen3d's makeCalcDataForTet / registerSideGCL and makeCalcDataForBoundary /
registerBoundarySideGCL with three coordinate levels, restated in
fp_set_moving_geometry) and the CPU restatement's GCL terms.

* three equal coordinate sets give the static arrays back bit for bit, with
  zero GCL weights;
* the discrete geometric conservation law that the solver checks
  (def_par:14590-14703) holds on every level for both time schemes: the GCL
  weights sum to the volume changes;
* a moving .sol round-trips;
* the residual of a uniform state is its GCL part to round-off, -q D / dt
  with D the volume change, for the central, LLF and Roe fluxes and both
  boundary terms (the HLLC flux takes half the interior part: it subtracts
  the GCL term of one state), and a uniform free stream stays uniform on a deforming mesh
  (single grid, timeScheme 2) to round-off: fluxes, GCL terms and time
  differences are consistent.
"""
import ctypes

import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, host_controls


def deform(x0, nb, t, boundary=False):
    """Smooth deformation of the interior nodes (and, with boundary, a rigid
    shift of every node) at time t."""
    d = np.zeros_like(x0)
    s = np.sin(np.pi * x0[0] / max(x0[0].max(), 1e-300))
    d[0] = 0.04 * np.sin(2 * np.pi * x0[1]) * s * np.sin(2 * np.pi * t)
    d[1] = 0.03 * np.sin(np.pi * x0[1]) * s * np.sin(2 * np.pi * t)
    d[2] = 0.02 * np.sin(np.pi * x0[2] / max(x0[2].max(), 1e-300)) * s * np.cos(2 * np.pi * t)
    d[:, :nb] = 0.0
    if boundary:
        d[1] += 0.05 * t
        d[2] -= 0.03 * t * t
    return x0 + d


@pytest.fixture
def mesh():
    m = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=3)
    yield m
    m.close()


def test_static_coordinates_give_static_arrays(mesh):
    names = ["side_w", "bnd_w", "volume", "side_len"]
    before = {(l, n): mesh.array(l, n) for l in (1, 2, 3) for n in names}
    rw = {l: mesh.array(l, "rweight") for l in (2, 3)}
    x0 = mesh.array(1, "coords")
    mesh.set_moving(x0, x0, x0, 2)
    for (l, n), a in before.items():
        assert np.array_equal(mesh.array(l, n), a), (l, n)
    for l in (2, 3):
        assert np.array_equal(mesh.array(l, "rweight"), rw[l])
    for l in (1, 2, 3):
        assert not np.any(mesh.array(l, "side_gcl")) and not np.any(mesh.array(l, "bnd_gcl"))
    assert np.array_equal(mesh.array(1, "volume_prev"), before[(1, "volume")])
    # the reader's second-order movement 1.5 x - 2 x + 0.5 x rounds to ~1 ulp
    assert np.abs(mesh.array(1, "coord_move")).max() < 1e-15


@pytest.mark.parametrize("boundary", [False, True])
@pytest.mark.parametrize("ts", [1, 2])
def test_geometric_conservation_law(mesh, ts, boundary):
    x0 = mesh.array(1, "coords")
    nb = mesh.level(1).n_bnodes
    mesh.set_moving(deform(x0, nb, 0.3, boundary), deform(x0, nb, 0.2, boundary), deform(x0, nb, 0.1, boundary), ts)
    for level in (1, 2, 3):
        err, scale = mesh.gcl_check(level, ts)
        assert scale > 1e-5, level  # the volumes do change
        assert err <= 1e-12 * scale, (level, err, scale)
    # the weights are those of a moving mesh: not zero, antisymmetric in use
    assert np.abs(mesh.array(1, "side_gcl")).max() > 1e-6
    if boundary:
        assert np.abs(mesh.array(1, "bnd_gcl")).max() > 1e-6
    # closure of the step's coefficients still holds
    closure, _ = mesh.check(1)
    assert closure < 1e-12


def test_coordinate_movement(mesh):
    x0 = mesh.array(1, "coords")
    nb = mesh.level(1).n_bnodes
    xs = [deform(x0, nb, t, True) for t in (0.3, 0.2, 0.1)]
    mesh.set_moving(*xs, 1)
    assert np.array_equal(mesh.array(1, "coord_move"), xs[0] - xs[1])
    mesh.set_moving(*xs, 2)
    assert np.array_equal(mesh.array(1, "coord_move"), (1.5 * xs[0] - 2.0 * xs[1]) + 0.5 * xs[2])
    assert np.array_equal(mesh.array(1, "coords"), xs[0])


def test_moving_sol_round_trip(mesh, tmp_path):
    x0 = mesh.array(1, "coords")
    nb = mesh.level(1).n_bnodes
    mesh.set_moving(deform(x0, nb, 0.3, True), deform(x0, nb, 0.2, True), deform(x0, nb, 0.1, True), 2)
    path = str(tmp_path / "moving.sol")
    mesh.write_sol(path)
    back = Mesh.read_sol(path)
    try:
        for level in (1, 2, 3):
            for name in ("side_w", "bnd_w", "volume", "side_gcl", "bnd_gcl"):
                assert np.array_equal(back.array(level, name), mesh.array(level, name)), (level, name)
        for name in ("volume_prev", "volume_prev2", "coords"):
            assert np.array_equal(back.array(1, name), mesh.array(1, name)), name
    finally:
        back.close()


def _oracle_case(mesh, ng=1, **ctl):
    base = dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=2.0, numberOfGridsToUse=ng, flowType=2,
                physicalTimeStep=0.1, timeScheme=2, MachNumber=0.5)
    c = host_controls(**{**base, **ctl})
    o = Solver(c, mesh, backend=oracle_backend())
    o.init_freestream()
    o.start()
    return c, o


@pytest.mark.parametrize("ctl", [dict(), dict(boundaryTerm=2), dict(fluxType=2), dict(fluxType=3),
                                 dict(fluxType=4), dict(timeScheme=1)])
def test_uniform_state_residual_is_its_gcl_part(ctl):
    # a flat channel: the free stream is tangential at the walls, so the
    # start's wall conditions leave it uniform
    mesh = Mesh.bump_channel(12, 4, 4, 0.0, nlevels=1)
    x0 = mesh.array(1, "coords")
    nb = mesh.level(1).n_bnodes
    ts = ctl.get("timeScheme", 2)
    mesh.set_moving(deform(x0, nb, 0.3, True), deform(x0, nb, 0.2, True), deform(x0, nb, 0.1, True), ts)
    c, o = _oracle_case(mesh, **ctl)
    try:
        u = np.ascontiguousarray(o.get_state(1))
        r = np.zeros_like(u)
        assert o.be.residual_fwd(o._h, 1, u.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p)) == 0
        V, Vp, Vp2 = (mesh.array(1, n) for n in ("volume", "volume_prev", "volume_prev2"))
        D = (1.5 * V - 2.0 * Vp) + 0.5 * Vp2 if ts == 2 else V - Vp
        # the GCL sums of the interior and of the boundary sides (the check
        # of def_par:14590-14610, with the reader's combination)
        comb = (lambda g, gp: 1.5 * g - 0.5 * gp) if ts == 2 else (lambda g, gp: g)
        sg, bg = mesh.array(1, "side_gcl"), mesh.array(1, "bnd_gcl")
        si, bi = mesh.array(1, "side_idx") - 1, mesh.array(1, "bnd_idx")[:2] - 1
        d_int, d_bnd = np.zeros_like(D), np.zeros_like(D)
        ww = comb(sg[0], sg[1])
        np.add.at(d_int, si[0], 2.0 * ww)
        np.add.at(d_int, si[1], -2.0 * ww)
        np.add.at(d_bnd, bi[0], 4.0 * comb(bg[0], bg[2]))
        np.add.at(d_bnd, bi[1], 4.0 * comb(bg[1], bg[3]))
        assert np.abs(d_int + d_bnd - D).max() <= 1e-12 * np.abs(D).max()
        # the HLLC flux subtracts the GCL term of one state (its wave
        # region's), the other fluxes that of both edge ends (def_par:1662-
        # 1791, 2074-2085): for a uniform state half the interior sum
        k = 0.5 if ctl.get("fluxType") == 4 else 1.0
        expect = -np.outer(u[:, 0], k * d_int + d_bnd) / c.physicalTimeStep
        assert np.abs(expect).max() > 1e-3
        static = _static_residual(mesh, u, **ctl)
        assert np.abs(static).max() < 1e-12
        assert np.abs(r - expect).max() <= 1e-11 * np.abs(expect).max()
    finally:
        o.close()
        mesh.close()


def _static_residual(mesh, u, **ctl):
    """The residual of u on the step's geometry without GCL terms."""
    base = dict(ReynoldsNumber=0.0, fluxType=1, numberOfGridsToUse=1, physicalTimeStep=0.1, MachNumber=0.5)
    c = host_controls(**{**base, **ctl, "flowType": 1})
    o = Solver(c, mesh, backend=oracle_backend())
    try:
        r = np.zeros_like(u)
        assert o.be.residual_fwd(o._h, 1, u.ctypes.data_as(ctypes.c_void_p), r.ctypes.data_as(ctypes.c_void_p)) == 0
        return r
    finally:
        o.close()


def test_free_stream_stays_uniform_on_a_deforming_mesh():
    mesh = Mesh.bump_channel(12, 4, 4, 0.0, nlevels=1)
    try:
        x0 = mesh.array(1, "coords")
        nb = mesh.level(1).n_bnodes
        dt = 0.1
        x = lambda k: deform(x0, nb, k * dt)
        mesh.set_moving(x(0), x(0), x(0), 2)
        c, o = _oracle_case(mesh, physicalTimeStep=dt)
        u_inf = o.get_state(1).copy()
        moved = 0.0
        for step in range(1, 5):
            if step > 1:
                o.next_physical_step()
            mesh.set_moving(x(step), x(step - 1), x(max(step - 2, 0)), 2)
            o.update_geometry(mesh)
            moved = max(moved, np.abs(x(step) - x0).max())
            for it in range(1, 4):
                o.cycle(it)
            assert np.abs(o.get_state(1) - u_inf).max() < 1e-12, step
        assert moved > 0.01
        o.close()
    finally:
        mesh.close()
