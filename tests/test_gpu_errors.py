"""Error paths and edge cases of the GPU library, each against the CPU
restatement where it has an answer: malformed level data, unsupported
controls, non-finite states, bad level numbers, the smallest mesh and more
grids requested than the mesh has."""
import ctypes

import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, _abi, default_controls, initial_state

pytestmark = pytest.mark.gpu

BASE = dict(ReynoldsNumber=0.0, fluxType=1, CFLNumber=2.0, multigridScheme=3)


def _create(c, descs, n):
    lib = _abi.gpu_lib()
    h = ctypes.c_void_p()
    rc = lib.flite_create(ctypes.byref(c), n, descs, ctypes.byref(h))
    if h:
        lib.flite_destroy(h)
    return rc


def _bad_descs(mesh, field, value_fn):
    # a copy of level 1's descriptor with one array replaced
    d = mesh.level(1)
    bad = _abi.LevelDesc.from_buffer_copy(d)
    arr = np.ascontiguousarray(value_fn(mesh.array(1, field)))
    setattr(bad, field, arr.ctypes.data_as(ctypes.c_void_p))
    descs = (_abi.LevelDesc * 1)(bad)
    return descs, arr  # keep arr alive


@pytest.mark.parametrize("field,fn", [
    ("side_idx", lambda a: np.where(np.arange(a.size).reshape(a.shape) == 7, 0, a).astype(np.int32)),
    ("side_idx", lambda a: np.where(np.arange(a.size).reshape(a.shape) == 3, a.max() + 5, a).astype(np.int32)),
    ("bnd_idx", lambda a: np.where(np.arange(a.size).reshape(a.shape) == 1, -2, a).astype(np.int32)),
])
def test_out_of_range_indices_are_rejected(field, fn):
    mesh = Mesh.bump_channel(4, 2, 2, 0.05, nlevels=1)
    c = default_controls(**BASE, numberOfGridsToUse=1)
    descs, keep = _bad_descs(mesh, field, fn)
    assert _create(c, descs, 1) == _abi.FLITE_EINVAL


@pytest.mark.parametrize("ctl,cpu_refuses", [
    (dict(turbulenceModel=2), True), (dict(flowType=3), True), (dict(flowType=2, physicalTimeStep=0.0), True),
    # moving meshes take the reference's fluxes, in FP64
    (dict(flowType=2, physicalTimeStep=0.1, reconstruction=1, fluxType=3), True),
    (dict(flowType=2, physicalTimeStep=0.1, precision=1), False),
    (dict(flowType=1, physicalTimeStep=0.0), True),
    (dict(viscosityScheme=3, ReynoldsNumber=100.0), True), (dict(coarseGridDissipationScheme=1), True),
    (dict(forceCalcType=2), True),
    (dict(fluxType=4, HLLCFluxOrder=2, GradientMethod=2, numberOfGridsToUse=2), True),
    # the extension's reconstruction belongs to the Roe flux; 3 or 5 stages
    (dict(reconstruction=1, fluxType=1), True), (dict(reconstruction=1, fluxType=4), True),
    (dict(reconstruction=2, fluxType=3), True), (dict(rungeKuttaStages=4), True),
    # FLITE_MIXED is a GPU-only mode, defined for the central flux alone
    (dict(precision=1, fluxType=4), False),
    (dict(precision=1, turbulenceModel=1, ReynoldsNumber=1e5), False),
])
def test_unsupported_controls_report_a_reason(ctl, cpu_refuses):
    mesh = Mesh.bump_channel(4, 2, 2, 0.05, nlevels=2)
    c = default_controls(**{**BASE, "numberOfGridsToUse": 2, **ctl})
    lib = _abi.gpu_lib()
    h = ctypes.c_void_p()
    assert lib.flite_create(ctypes.byref(c), mesh.nlevels, mesh.descs, ctypes.byref(h)) == _abi.FLITE_EUNSUPPORTED
    assert not h
    buf = ctypes.create_string_buffer(256)
    lib.flite_last_error(None, buf, len(buf))
    assert buf.value
    if cpu_refuses:
        with pytest.raises(RuntimeError, match="status 2"):
            Solver(c, mesh, backend=oracle_backend())


def test_non_finite_state_reports_enan():
    mesh = Mesh.bump_channel(6, 2, 2, 0.05, nlevels=2)
    c = default_controls(**BASE, numberOfGridsToUse=2)
    s = Solver(c, mesh)
    u = initial_state(c, mesh)
    u[0, 3] = np.nan
    s.set_state(u)
    s.start()
    s.cycle(1)
    with pytest.raises(FloatingPointError):
        s.residuals()


def test_bad_level_numbers_are_rejected():
    mesh = Mesh.bump_channel(6, 2, 2, 0.05, nlevels=2)
    c = default_controls(**BASE, numberOfGridsToUse=2)
    s = Solver(c, mesh)
    lib = _abi.gpu_lib()
    buf = np.zeros(5 * mesh.level(1).n_nodes)
    for level in (0, 3, -1):
        assert lib.flite_get_state(s._h, level, buf.ctypes.data_as(ctypes.c_void_p)) == _abi.FLITE_EINVAL
        assert lib.flite_do_time_iterations(s._h, level, 1, 1, 0, 1) == _abi.FLITE_EINVAL
    assert lib.flite_prolong(s._h, 1) == _abi.FLITE_EINVAL
    assert lib.flite_restrict(s._h, 2, 0) == _abi.FLITE_EINVAL


@pytest.mark.parametrize("ctl", [dict(), dict(ReynoldsNumber=500.0, wallsAreIsentropic=1),
                                 dict(fluxType=4, HLLCFluxOrder=2, Automaticlipping=1)])
def test_smallest_mesh_matches_restatement(ctl):
    # one hex split into six tets: every node is a boundary node
    mesh = Mesh.bump_channel(1, 1, 1, 0.0, nlevels=1)
    c = default_controls(**{**BASE, "numberOfGridsToUse": 1, "CFLNumber": 0.5, **ctl})
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    u0 = initial_state(c, mesh, perturb_seed=1, amplitude=0.05)
    for s in (g, o):
        s.set_state(u0)
        s.start()
    for cyc in range(1, 4):
        g.cycle(cyc)
        o.cycle(cyc)
    assert np.array_equal(g.get_state(1), o.get_state(1))


def test_more_grids_requested_than_the_mesh_has():
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=2)
    c = default_controls(**BASE, numberOfGridsToUse=5)
    g, o = Solver(c, mesh), Solver(c, mesh, backend=oracle_backend())
    assert g.nlevels == 2
    u0 = initial_state(c, mesh, perturb_seed=3)
    for s in (g, o):
        s.set_state(u0)
        s.start()
    for cyc in range(1, 3):
        g.cycle(cyc)
        o.cycle(cyc)
    assert np.array_equal(g.get_state(2), o.get_state(2))
