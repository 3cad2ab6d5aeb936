"""The residual entry point that allocates nothing (flite_residual_noalloc).

It serves callers that cannot call cudaMalloc, such as a host whose device
memory belongs to another allocator; its scratch is a static device array
inside the library.  Its output must equal flite_residual_fwd's, bit for bit
(the tolerance of the other parity tests of the FP64 path), on two calls in a
row -- the second call reuses the scratch the first one left behind.  The
test allocates its own device arrays with torch; the entry point does not.
"""
import ctypes

import numpy as np
import pytest

from flite3d_b200 import Mesh, Solver, _abi, default_controls, initial_state

pytestmark = pytest.mark.gpu


class _BoundaryCodesView:
    """A one-level mesh whose boundary-edge array is replaced (other codes on
    some faces), with the descriptors Solver reads."""

    def __init__(self, mesh, bnd_idx):
        self._keep = np.asfortranarray(bnd_idx, dtype=np.int32).copy()
        self.nlevels = 1
        self.descs = (_abi.LevelDesc * 1)(mesh.level(1))
        self.descs[0].bnd_idx = self._keep.ctypes.data_as(ctypes.c_void_p)

    def level(self, level):
        return self.descs[level - 1]


def _call(lib, c, n, e, b, side_idx, side_w, bnd_idx, bnd_w, u, rhs):
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    return lib.flite_residual_noalloc(ctypes.byref(c), n, e, b, p(side_idx), p(side_w), p(bnd_idx), p(bnd_w),
                                      p(u), p(rhs), None)


def _dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_noalloc_matches_residual_fwd_twice(gpu):
    import torch
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=1)
    c = default_controls(ReynoldsNumber=0.0, fluxType=1)
    solver = Solver(c, mesh)
    d = mesh.level(1)
    n, e, b = d.n_nodes, d.n_sides, d.n_bsides
    side_idx = _dev(mesh.array(1, "side_idx"), torch)
    side_w = _dev(mesh.array(1, "side_w"), torch)
    bnd_idx = _dev(mesh.array(1, "bnd_idx"), torch)
    bnd_w = _dev(mesh.array(1, "bnd_w"), torch)
    lib = _abi.gpu_lib()
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    for seed in (3, 11):
        u = initial_state(c, mesh, perturb_seed=seed, amplitude=0.05)
        u[1] *= 1.0 + 0.03 * np.cos(np.arange(n) * seed)
        du = _dev(u, torch)
        rhs = torch.full((5, n), np.nan, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.flite_residual_noalloc(ctypes.byref(c), n, e, b, ptr(side_idx), ptr(side_w),
                                        ptr(bnd_idx), ptr(bnd_w), ptr(du), ptr(rhs), None)
        assert rc == _abi.FLITE_OK
        torch.cuda.synchronize()
        expect = solver.residual_fwd(u)
        assert np.array_equal(rhs.cpu().numpy(), expect)


def test_noalloc_rejects_oversize(gpu):
    import torch
    c = default_controls(ReynoldsNumber=0.0, fluxType=1)
    lib = _abi.gpu_lib()
    x = torch.zeros(16, dtype=torch.float64, device="cuda")
    i = torch.ones(16, dtype=torch.int32, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = lib.flite_residual_noalloc(ctypes.byref(c), 65537, 1, 0, p(i), p(x), p(i), p(x), p(x),
                                    p(x), None)
    assert rc == _abi.FLITE_EINVAL


def test_noalloc_far_field_code_4_matches_residual_fwd(gpu):
    # far-field faces of code 4 read the second freestream set,
    # inflowField[6..11]; make it differ from the first
    import torch
    mesh = Mesh.bump_channel(12, 4, 4, 0.05, nlevels=1)
    c = default_controls(ReynoldsNumber=0.0, fluxType=1)
    c.inflowField[6 + 0] = 1.05
    c.inflowField[6 + 5] = c.inflowField[5] * 0.97
    bidx = mesh.array(1, "bnd_idx")
    xyz = mesh.array(1, "coords")
    outflow = (bidx[2] == 3) & (xyz[0, bidx[0] - 1] > 2.999)
    assert outflow.any()
    bidx[2, outflow] = 4
    view = _BoundaryCodesView(mesh, bidx)
    solver = Solver(c, view)
    n, e, b = mesh.level(1).n_nodes, mesh.level(1).n_sides, mesh.level(1).n_bsides
    dev = lambda a: _dev(a, torch)  # noqa: E731
    side_idx, side_w = dev(mesh.array(1, "side_idx")), dev(mesh.array(1, "side_w"))
    bnd_idx, bnd_w = dev(bidx), dev(mesh.array(1, "bnd_w"))
    u = initial_state(c, mesh, perturb_seed=5, amplitude=0.05)
    du = dev(u)
    rhs = torch.full((5, n), np.nan, dtype=torch.float64, device="cuda")
    assert _call(_abi.gpu_lib(), c, n, e, b, side_idx, side_w, bnd_idx, bnd_w, du, rhs) == _abi.FLITE_OK
    torch.cuda.synchronize()
    assert np.array_equal(rhs.cpu().numpy(), solver.residual_fwd(u))


def test_noalloc_refuses_bad_indices_and_codes_as_create_does(gpu):
    import torch
    mesh = Mesh.bump_channel(8, 4, 4, 0.05, nlevels=1)
    c = default_controls(ReynoldsNumber=0.0, fluxType=1)
    n, e, b = mesh.level(1).n_nodes, mesh.level(1).n_sides, mesh.level(1).n_bsides
    dev = lambda a: _dev(a, torch)  # noqa: E731
    sidx, bidx = mesh.array(1, "side_idx"), mesh.array(1, "bnd_idx")
    side_w, bnd_w = dev(mesh.array(1, "side_w")), dev(mesh.array(1, "bnd_w"))
    u = dev(initial_state(c, mesh))
    rhs = torch.zeros((5, n), dtype=torch.float64, device="cuda")
    lib = _abi.gpu_lib()
    # node indices outside 1..N: the kernel drops the edge, the call says EINVAL
    for bad in (0, n + 1):
        s2 = sidx.copy()
        s2[1, 7] = bad
        assert _call(lib, c, n, e, b, dev(s2), side_w, dev(bidx), bnd_w, u, rhs) == _abi.FLITE_EINVAL
    # boundary codes outside 1..9
    for bad in (0, 10):
        b2 = bidx.copy()
        b2[2, 3] = bad
        assert _call(lib, c, n, e, b, dev(sidx), side_w, dev(b2), bnd_w, u, rhs) == _abi.FLITE_EINVAL
    # an engine face (codes 5..8) takes the engine flux, as in residual_fwd
    b5 = bidx.copy()
    b5[2, 3] = 5
    b5[2, 9] = 8
    assert _call(lib, c, n, e, b, dev(sidx), side_w, dev(b5), bnd_w, u, rhs) == _abi.FLITE_OK
    torch.cuda.synchronize()
    engine_view = Solver(c, _BoundaryCodesView(mesh, b5))
    assert np.array_equal(rhs.cpu().numpy(), engine_view.residual_fwd(u.cpu().numpy()))
    engine_view.close()
    # the entry point still works after the refusals
    good = torch.full((5, n), np.nan, dtype=torch.float64, device="cuda")
    assert _call(lib, c, n, e, b, dev(sidx), side_w, dev(bidx), bnd_w, u, good) == _abi.FLITE_OK


def test_noalloc_without_edges_gives_a_zero_residual(gpu):
    # no interior and no boundary edges: nothing to sum, every node's residual 0
    import torch
    c = default_controls(ReynoldsNumber=0.0, fluxType=1)
    lib = _abi.gpu_lib()
    n = 5
    u = torch.ones((5, n), dtype=torch.float64, device="cuda")
    rhs = torch.full((5, n), np.nan, dtype=torch.float64, device="cuda")
    i = torch.ones(2, dtype=torch.int32, device="cuda")
    w = torch.zeros(3, dtype=torch.float64, device="cuda")
    assert _call(lib, c, n, 0, 0, i, w, i, w, u, rhs) == _abi.FLITE_OK
    torch.cuda.synchronize()
    assert np.array_equal(rhs.cpu().numpy(), np.zeros((5, n)))
