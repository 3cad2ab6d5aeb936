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
