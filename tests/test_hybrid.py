"""Hybrid elements on the CPU: the median-dual coefficients and volumes of
hexahedra, prisms and pyramids (makeCalcDataForHex / Pri / Pyr,
gen3d_grid.f90:902-2090) and of quadrilateral boundary faces
(makeCalcDataForBoundary, gen3d_boundary.f90:627-766), restated in
fp_from_elements.

* the dual of a box meshed with each element type, and with columns of all
  three, closes at every node and its volumes sum to the box's volume (the
  same as the tetrahedral split's);
* on a deforming hybrid mesh the discrete geometric conservation law holds on
  every level (the element routines' GCL terms);
* a uniform stream along the box's flat walls is a steady state of the CPU
  restatement on every such mesh (residual at round-off).
"""
import ctypes

import numpy as np
import pytest

from conftest import oracle_backend
from flite3d_b200 import Mesh, Solver, host_controls
from hybrid_meshes import VOLUME, box

KINDS = ["hex", "prism", "pyramid", "mixed"]


@pytest.mark.parametrize("kind", KINDS)
def test_dual_closes_and_fills_the_box(kind):
    m = box(kind=kind, nlevels=2)
    try:
        closure, vol = m.check(1)
        assert closure < 1e-14
        assert abs(vol - VOLUME) < 1e-12
        assert np.all(m.array(1, "volume") > 0)
        # the coarse level sums the fine volumes
        assert abs(m.check(2)[1] - VOLUME) < 1e-12
    finally:
        m.close()


def test_hexahedra_and_their_tetrahedral_split_fill_the_same_volume():
    # the same box as six tetrahedra per hexahedron (fp_from_tets)
    import hybrid_meshes as H
    nx, ny, nz = 6, 3, 3
    xyz = H._grid(nx, ny, nz)
    hexm = box(nx, ny, nz, "hex")
    tets = []
    for h in _hexes(nx, ny, nz):
        for t in ((0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)):
            tets.append([h[t[0]], h[t[1]], h[t[2]], h[t[3]]])
    tris, ind = [], []
    for q, i in _box_quads(nx, ny, nz):
        tris += [[q[0], q[1], q[2]], [q[0], q[2], q[3]]]
        ind += [i, i]
    tetm = Mesh.from_tets(xyz, tets, tris, ind, nlevels=1)
    try:
        assert abs(tetm.check(1)[1] - hexm.check(1)[1]) < 1e-12
        assert hexm.sizes(1)["nodes"] == tetm.sizes(1)["nodes"]
    finally:
        tetm.close()
        hexm.close()


def _nid(ny, nz):
    return lambda i, j, k: (i * (ny + 1) + j) * (nz + 1) + k + 1


def _hexes(nx, ny, nz):
    nid = _nid(ny, nz)
    return [[nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
             nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)]
            for i in range(nx) for j in range(ny) for k in range(nz)]


def _box_quads(nx, ny, nz):
    nid = _nid(ny, nz)
    out = []
    for i in range(nx):
        for j in range(ny):
            out.append(([nid(i, j, 0), nid(i + 1, j, 0), nid(i + 1, j + 1, 0), nid(i, j + 1, 0)], 1))
            out.append(([nid(i, j, nz), nid(i + 1, j, nz), nid(i + 1, j + 1, nz), nid(i, j + 1, nz)], 2))
        for k in range(nz):
            for j in (0, ny):
                out.append(([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j, k + 1), nid(i, j, k + 1)], 2))
    for j in range(ny):
        for k in range(nz):
            for i in (0, nx):
                out.append(([nid(i, j, k), nid(i, j + 1, k), nid(i, j + 1, k + 1), nid(i, j, k + 1)], 3))
    return out


@pytest.mark.parametrize("ts", [1, 2])
@pytest.mark.parametrize("kind", KINDS)
def test_geometric_conservation_law_on_hybrid_meshes(kind, ts):
    m = box(kind=kind, nlevels=2)
    try:
        x0 = m.array(1, "coords")
        nb = m.level(1).n_bnodes

        def x(t):
            d = 0.05 * np.sin(np.pi * x0[0] / 3.0) * np.sin(np.pi * x0[1]) * np.sin(np.pi * x0[2]) * t
            y = x0.copy()
            y[0, nb:] += d[nb:]
            y[2, nb:] -= 0.5 * d[nb:]
            y[1] += 0.03 * t
            return y
        m.set_moving(x(0.3), x(0.2), x(0.05), ts)
        for level in (1, 2):
            err, scale = m.gcl_check(level, ts)
            assert scale > 1e-5 and err <= 1e-12 * scale, (level, err, scale)
    finally:
        m.close()


@pytest.mark.parametrize("kind", KINDS)
def test_uniform_stream_is_steady(kind):
    m = box(kind=kind, nlevels=1)
    try:
        c = host_controls(ReynoldsNumber=0.0, fluxType=1, MachNumber=0.5, numberOfGridsToUse=1)
        o = Solver(c, m, backend=oracle_backend())
        o.init_freestream()
        o.start()
        u = np.ascontiguousarray(o.get_state(1))
        r = o.residual_fwd(u)
        assert np.abs(r).max() < 1e-13
        o.close()
    finally:
        m.close()
