"""Structured boxes of gen3d's element types for the tests: a sheared box
(planar faces, volume 3) of hexahedra, of prisms (each hexahedron split along
its diagonal plane 1-3-7-5), of pyramids (six per hexahedron around a centre
node), of columns of hexahedra and prisms, or of tetrahedra (six per
hexahedron around its diagonal 1-7, triangular boundary faces).  Walls at
z = 0 (indicator 1), symmetry at y = const and z = 1 (2), far field at
x = const (3).  With engines, the inner faces of the outflow plane x = 3 are
engine inlets (indicator 5 where y < 1/2, 6 above; 5 throughout with one
engine) and those of the inflow plane x = 0 engine exhausts (7 and 8
alike)."""
import numpy as np

from flite3d_b200 import Mesh

VOLUME = 3.0


def _grid(nx, ny, nz):
    ii, jj, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    x = ii / nx * 3.0 + 0.2 * jj / ny
    y = jj / ny * 1.0 + 0.1 * kk / nz
    z = kk / nz * 1.0
    return np.stack([x.ravel(), y.ravel(), z.ravel()], 1)


def _lowest_first(q):
    """A quadrilateral from its lowest-numbered vertex on: the diagonal 1-3
    that a pyramid base and a boundary face take is then the same for every
    element sharing the face."""
    k = int(np.argmin(q))
    return q[k:] + q[:k]


def box(nx=6, ny=3, nz=3, kind="hex", nlevels=2, engines=False, far_only=False):
    """kind: "hex", "prism", "pyramid", "mixed" (columns of hexahedra and
    prisms, whose face diagonals follow the node numbers alike) or "tet";
    far_only (tetrahedra): every face that is not an engine face is far field."""
    if kind == "tet":
        return _tet_box(nx, ny, nz, nlevels, engines, far_only)
    xyz = _grid(nx, ny, nz)

    def nid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k + 1

    def kind_of(i, j):
        return kind if kind != "mixed" else ("hex", "prism")[(i + j) % 2]

    hexes, prisms, pyramids, centres = [], [], [], []
    tris, tind, quads, qind = [], [], [], []
    n0 = xyz.shape[0]
    for i in range(nx):
        for j in range(ny):
            kd = kind_of(i, j)
            for k in range(nz):
                h = [nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                     nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)]
                if kd == "hex":
                    hexes.append(h)
                elif kd == "prism":
                    prisms.append([h[0], h[1], h[2], h[4], h[5], h[6]])
                    prisms.append([h[0], h[2], h[3], h[4], h[6], h[7]])
                else:
                    c = n0 + len(centres) + 1
                    centres.append(xyz[np.array(h) - 1].mean(0))
                    for f in ((0, 1, 2, 3), (7, 6, 5, 4), (0, 4, 5, 1), (1, 5, 6, 2), (2, 6, 7, 3), (3, 7, 4, 0)):
                        pyramids.append(_lowest_first([h[f[0]], h[f[1]], h[f[2]], h[f[3]]]) + [c])
            # z faces: triangles under prisms, quadrilaterals otherwise
            for k, ind in ((0, 1), (nz, 2)):
                q = [nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k)]
                if kd == "prism":
                    tris += [[q[0], q[1], q[2]], [q[0], q[2], q[3]]]
                    tind += [ind, ind]
                else:
                    quads.append(_lowest_first(q))
                    qind.append(ind)
    for i in range(nx):
        for k in range(nz):
            for j in (0, ny):
                quads.append(_lowest_first([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j, k + 1), nid(i, j, k + 1)]))
                qind.append(2)
    for j in range(ny):
        for k in range(nz):
            for i in (0, nx):
                quads.append(_lowest_first([nid(i, j, k), nid(i, j + 1, k), nid(i, j + 1, k + 1), nid(i, j, k + 1)]))
                qind.append(_x_face_indicator(i == nx, j, k, ny, nz, engines))
    if centres:
        xyz = np.concatenate([xyz, np.array(centres)])
    return Mesh.from_elements(xyz, hexes=hexes, prisms=prisms, pyramids=pyramids, tris=tris, tri_indicator=tind,
                              quads=quads, quad_indicator=qind, nlevels=nlevels)


def _x_face_indicator(outflow, j, k, ny, nz, engines):
    """Far field, or on the inner faces of the x planes the engine inlets
    (outflow plane) and exhausts (inflow plane) of engines 1 and 2."""
    if engines and 1 <= j < ny - 1 and 1 <= k < nz - 1:
        engine = 1 if j < ny // 2 or engines == 1 else 2
        return 4 + engine if outflow else 6 + engine
    return 3


def _tet_box(nx, ny, nz, nlevels, engines, far_only=False):
    xyz = _grid(nx, ny, nz)

    def nid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k + 1

    tets, tris, ind = [], [], []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                h = [nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                     nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)]
                for t in ((0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)):
                    tets.append([h[t[0]], h[t[1]], h[t[2]], h[t[3]]])

    def quad(q, indicator):  # split along q0-q2, the diagonal of the tetrahedra
        if far_only and indicator in (1, 2):
            indicator = 3
        tris.extend([[q[0], q[1], q[2]], [q[0], q[2], q[3]]])
        ind.extend([indicator, indicator])

    for i in range(nx):
        for j in range(ny):
            quad([nid(i, j, 0), nid(i + 1, j, 0), nid(i + 1, j + 1, 0), nid(i, j + 1, 0)], 1)
            quad([nid(i, j, nz), nid(i + 1, j, nz), nid(i + 1, j + 1, nz), nid(i, j + 1, nz)], 2)
        for k in range(nz):
            for j in (0, ny):
                quad([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j, k + 1), nid(i, j, k + 1)], 2)
    for j in range(ny):
        for k in range(nz):
            for i in (0, nx):
                quad([nid(i, j, k), nid(i, j + 1, k), nid(i, j + 1, k + 1), nid(i, j, k + 1)],
                     _x_face_indicator(i == nx, j, k, ny, nz, engines))
    return Mesh.from_tets(xyz, tets, tris, ind, nlevels=nlevels)
