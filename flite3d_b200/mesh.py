"""Meshes and reference file formats (wraps libflite_prepro.so).

A :class:`Mesh` holds the multi-level solver input that gen3d writes to a
``.sol`` file (PreProSource/gen3d_grid.f90:4082-5231) and hands the
solver one :class:`~flite3d_b200._abi.LevelDesc` per level, exactly the
arrays readGridComputationData reads (SolverSource/mgnsg3d_def_par.F90:
13812-14074).
"""
import ctypes

import numpy as np

from . import _abi

_c_double = ctypes.c_double


def _lib():
    return _abi.prepro_lib()


class Mesh:
    """Multi-level mesh owned by the preprocessor library."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle) if not isinstance(handle, ctypes.c_void_p) else handle
        self.nlevels = _lib().fp_num_levels(self._h)
        self._descs = (_abi.LevelDesc * self.nlevels)()
        self._refresh()

    def _refresh(self):
        for level in range(self.nlevels):
            _abi.check(_lib().fp_level_desc(self._h, level + 1, ctypes.byref(self._descs[level])),
                       "fp_level_desc")

    # ---- construction -------------------------------------------------
    @classmethod
    def bump_channel(cls, nx, ny, nz, bump_height=0.05, nlevels=3):
        """Bump channel [0,3]x[0,1]x[0,1], nx*ny*nz hexes split into 6 tets."""
        h = ctypes.c_void_p()
        _abi.check(_lib().fp_bump_channel(int(nx), int(ny), int(nz), _c_double(bump_height),
                                          int(nlevels), ctypes.byref(h)), "fp_bump_channel")
        return cls(h)

    @classmethod
    def naca0012(cls, ni, nj, nk, first_cell=1.0e-5, growth=1.15, nlayer=40, farfield=20.0, span=1.0,
                 nlevels=3):
        """Extruded NACA0012 O-grid (wall 1, span ends 2, far field 3)."""
        h = ctypes.c_void_p()
        _abi.check(_lib().fp_naca0012(int(ni), int(nj), int(nk), ctypes.c_double(first_cell),
                                      ctypes.c_double(growth), int(nlayer), ctypes.c_double(farfield),
                                      ctypes.c_double(span), int(nlevels), ctypes.byref(h)), "fp_naca0012")
        return cls(h)

    @classmethod
    def from_tets(cls, xyz, tets, tris, tri_indicator, nlevels=3):
        """xyz (N,3), tets (T,4), tris (F,3) 1-based, indicators (F,) in 1..9."""
        xyz = np.asfortranarray(np.asarray(xyz, dtype=np.float64))
        tets = np.asfortranarray(np.asarray(tets, dtype=np.int32))
        tris = np.asfortranarray(np.asarray(tris, dtype=np.int32))
        ind = np.ascontiguousarray(np.asarray(tri_indicator, dtype=np.int32))
        h = ctypes.c_void_p()
        _abi.check(_lib().fp_from_tets(
            xyz.shape[0], xyz.ctypes.data_as(ctypes.c_void_p), tets.shape[0],
            tets.ctypes.data_as(ctypes.c_void_p), tris.shape[0],
            tris.ctypes.data_as(ctypes.c_void_p), ind.ctypes.data_as(ctypes.c_void_p),
            int(nlevels), ctypes.byref(h)), "fp_from_tets")
        return cls(h)

    @classmethod
    def from_elements(cls, xyz, tets=None, pyramids=None, prisms=None, hexes=None, tris=None, tri_indicator=None,
                      quads=None, quad_indicator=None, nlevels=3):
        """A mesh of hybrid elements: xyz (N, 3); tets (n, 4), pyramids
        (n, 5), prisms (n, 6), hexes (n, 8); boundary tris (n, 3) and quads
        (n, 4) with indicators; 1-based node numbers."""
        xyz = np.asfortranarray(np.asarray(xyz, dtype=np.float64))
        keep = []

        def arr(a, k):
            if a is None or len(a) == 0:
                return 0, None
            v = np.asfortranarray(np.asarray(a, dtype=np.int32).reshape(-1, k))
            keep.append(v)
            return v.shape[0], v.ctypes.data_as(ctypes.c_void_p)

        def ind(a):
            if a is None or len(a) == 0:
                return None
            v = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
            keep.append(v)
            return v.ctypes.data_as(ctypes.c_void_p)
        nt, pt = arr(tets, 4)
        ny, py = arr(pyramids, 5)
        npr, pp = arr(prisms, 6)
        nh, ph = arr(hexes, 8)
        nf, pf = arr(tris, 3)
        nq, pq = arr(quads, 4)
        h = ctypes.c_void_p()
        _abi.check(_lib().fp_from_elements(xyz.shape[0], xyz.ctypes.data_as(ctypes.c_void_p), nt, pt, ny, py, npr, pp,
                                           nh, ph, nf, pf, ind(tri_indicator), nq, pq, ind(quad_indicator),
                                           int(nlevels), ctypes.byref(h)), "fp_from_elements")
        return cls(h)

    @classmethod
    def read_sol(cls, path):
        h = ctypes.c_void_p()
        _abi.check(_lib().fp_read_sol(str(path).encode(), ctypes.byref(h)), "fp_read_sol")
        return cls(h)

    def write_sol(self, path):
        _abi.check(_lib().fp_write_sol(self._h, str(path).encode()), "fp_write_sol")

    @classmethod
    def read_sol_domains(cls, prefix, plotreg):
        """The mesh of a parallel run's files prefix.sol_1.. with plotreg,
        merged into one (canonical form)."""
        h = ctypes.c_void_p()
        _abi.check(_lib().fp_read_sol_domains(str(prefix).encode(), str(plotreg).encode(), ctypes.byref(h)),
                   "fp_read_sol_domains")
        return cls(h)

    def partition(self, ndomains):
        """gen3d's greedy partition of level 1: the 1-based domain of every
        node (N,)."""
        col = np.zeros(self.level(1).n_nodes, dtype=np.int32)
        n = ctypes.c_int32()
        _abi.check(_lib().fp_partition(self._h, int(ndomains), col.ctypes.data_as(ctypes.c_void_p),
                                       ctypes.byref(n)), "fp_partition")
        return col

    def write_sol_domains(self, prefix, plotreg, ndomains, color=None):
        """The files of a parallel run over ndomains (or the given 1-based
        level-1 domains): prefix.sol_1.. and plotreg."""
        c = None if color is None else np.ascontiguousarray(color, dtype=np.int32)
        _abi.check(_lib().fp_write_sol_domains(self._h, str(prefix).encode(), str(plotreg).encode(), int(ndomains),
                                               None if c is None else c.ctypes.data_as(ctypes.c_void_p)),
                   "fp_write_sol_domains")

    def canonical(self):
        """The canonical form of this mesh (a new Mesh)."""
        h = ctypes.c_void_p()
        _abi.check(_lib().fp_canonical(self._h, ctypes.byref(h)), "fp_canonical")
        return Mesh(h)

    def write_plt(self, path):
        _abi.check(_lib().fp_write_plt(self._h, str(path).encode()), "fp_write_plt")

    def write_plotreg(self, path):
        _abi.check(_lib().fp_write_plotreg(self._h, str(path).encode()), "fp_write_plotreg")

    def close(self):
        if self._h:
            _lib().fp_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- access --------------------------------------------------------
    @property
    def descs(self):
        return self._descs

    def level(self, level):
        return self._descs[level - 1]

    def sizes(self, level=1):
        d = self.level(level)
        return dict(nodes=d.n_nodes, sides=d.n_sides, bsides=d.n_bsides, bnodes=d.n_bnodes)

    def check(self, level=1):
        closure, vol = _c_double(), _c_double()
        _abi.check(_lib().fp_check(self._h, level, ctypes.byref(closure), ctypes.byref(vol)),
                   "fp_check")
        return closure.value, vol.value

    def geometry(self, xyz=None):
        """Level-1 side_w (3, E), bnd_w (3, B) and volume (N) of the mesh's
        own elements at the node coordinates xyz (3, N) (None: the mesh's)."""
        d = self.level(1)
        sw = np.zeros((3, d.n_sides)); bw = np.zeros((3, d.n_bsides)); vol = np.zeros(d.n_nodes)
        x = None if xyz is None else np.ascontiguousarray(xyz, dtype=np.float64)
        _abi.check(_lib().fp_geometry(self._h, None if x is None else x.ctypes.data_as(ctypes.c_void_p),
                                      sw.ctypes.data_as(ctypes.c_void_p), bw.ctypes.data_as(ctypes.c_void_p),
                                      vol.ctypes.data_as(ctypes.c_void_p)), "fp_geometry")
        return sw, bw, vol

    def geometry_vjp(self, side_w_bar, bnd_w_bar, volume_bar, xyz=None):
        """(d geometry / d xyz)^T applied to the three geometry adjoints:
        the sensitivity (3, N) of a function of the level-1 geometry to the
        node coordinates."""
        d = self.level(1)
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (side_w_bar, bnd_w_bar, volume_bar)]
        xb = np.zeros((3, d.n_nodes))
        x = None if xyz is None else np.ascontiguousarray(xyz, dtype=np.float64)
        _abi.check(_lib().fp_geometry_vjp(self._h, None if x is None else x.ctypes.data_as(ctypes.c_void_p),
                                          *[v.ctypes.data_as(ctypes.c_void_p) for v in a],
                                          xb.ctypes.data_as(ctypes.c_void_p)), "fp_geometry_vjp")
        return xb

    def set_moving(self, xyz, xyz_prev, xyz_prev2, time_scheme=2):
        """Moving meshes (flowType 2): the geometry of every level for the
        physical step with node coordinates xyz, the two steps before having
        had xyz_prev and xyz_prev2 (each (3, N)); the descriptors then carry
        the GCL weights, previous volumes and coordinate movement."""
        xs = [np.ascontiguousarray(x, dtype=np.float64) for x in (xyz, xyz_prev, xyz_prev2)]
        _abi.check(_lib().fp_set_moving_geometry(self._h, *[x.ctypes.data_as(ctypes.c_void_p) for x in xs],
                                                 int(time_scheme)), "fp_set_moving_geometry")
        self._refresh()

    def gcl_check(self, level=1, time_scheme=2):
        """(largest GCL defect, largest volume change) of a moving level."""
        err, scale = _c_double(), _c_double()
        _abi.check(_lib().fp_gcl_check(self._h, level, int(time_scheme), ctypes.byref(err), ctypes.byref(scale)),
                   "fp_gcl_check")
        return err.value, scale.value

    def with_level1_geometry(self, side_w, bnd_w, volume):
        """Level descriptors of this mesh with level 1's side_w, bnd_w and
        volume replaced (the arrays are kept alive by the returned object,
        which has the nlevels / descs / level() of a Mesh for Solver)."""
        return _GeometryView(self, side_w, bnd_w, volume)

    def array(self, level, name):
        """Copy of one level array as numpy (column-major fields as (k, n))."""
        d = self.level(level)
        n, e, b = d.n_nodes, d.n_sides, d.n_bsides
        spec = {
            "side_idx": (d.side_idx, np.int32, (2, e)), "side_w": (d.side_w, np.float64, (3, e)),
            "side_len": (d.side_len, np.float64, (e,)), "bnd_idx": (d.bnd_idx, np.int32, (3, b)),
            "bnd_w": (d.bnd_w, np.float64, (3, b)), "node_reg": (d.node_reg, np.int32, (21,)),
            "node_ind": (d.node_ind, np.int32, (d.n_normals,)),
            "volume": (d.volume, np.float64, (n,)), "wall_dist": (d.wall_dist, np.float64, (n,)),
            "coords": (d.coords, np.float64, (3, n)), "coord_move": (d.coord_move, np.float64, (3, n)),
            "side_gcl": (d.side_gcl, np.float64, (2, e)), "bnd_gcl": (d.bnd_gcl, np.float64, (4, b)),
            "volume_prev": (d.volume_prev, np.float64, (n,)), "volume_prev2": (d.volume_prev2, np.float64, (n,)),
            "engine_idx": (d.engine_idx, np.int32, (3, d.n_engine_sides)),
            "engine_w": (d.engine_w, np.float64, (3, d.n_engine_sides)),
        }
        if level > 1:
            nf = self.level(level - 1).n_nodes
            spec["parent"] = (d.parent, np.int32, (nf,))
            spec["rweight"] = (d.rweight, np.float64, (nf,))
        ptr, dt, shape = spec[name]
        if not ptr:
            return None
        count = int(np.prod(shape))
        ctype = ctypes.c_int32 if dt == np.int32 else ctypes.c_double
        buf = (ctype * count).from_address(ptr)
        return np.frombuffer(buf, dtype=dt, count=count).reshape(shape).copy()


class _GeometryView:
    """A mesh whose level-1 geometry arrays are replaced (perturbed meshes of
    finite-difference checks, moved surfaces)."""

    def __init__(self, mesh, side_w, bnd_w, volume):
        self.mesh = mesh
        self._keep = [np.ascontiguousarray(a, dtype=np.float64) for a in (side_w, bnd_w, volume)]
        self.nlevels = mesh.nlevels
        self.descs = (_abi.LevelDesc * mesh.nlevels)(*[mesh.level(l + 1) for l in range(mesh.nlevels)])
        d = self.descs[0]
        d.side_w, d.bnd_w, d.volume = [a.ctypes.data_as(ctypes.c_void_p) for a in self._keep]

    def level(self, level):
        return self.descs[level - 1]

    def array(self, level, name):
        return self.mesh.array(level, name)


# ---- restart / result files ---------------------------------------------

def write_rst(path, prim):
    """prim: (nvar, N) primitive rho, u, v, w, E/rho [, nu] (def_par:3740-3873)."""
    prim = np.ascontiguousarray(prim, dtype=np.float64)
    nvar, n = prim.shape
    _abi.check(_lib().fp_write_rst(str(path).encode(), n, nvar, prim.ctypes.data_as(ctypes.c_void_p)),
               "fp_write_rst")


def read_rst(path, n, nvar=5):
    out = np.zeros((nvar, n))
    _abi.check(_lib().fp_read_rst(str(path).encode(), n, nvar, out.ctypes.data_as(ctypes.c_void_p)),
               "fp_read_rst")
    return out


def write_res(path, u):
    u = np.ascontiguousarray(u, dtype=np.float64)
    nvar, n = u.shape
    _abi.check(_lib().fp_write_res(str(path).encode(), n, nvar, u.ctypes.data_as(ctypes.c_void_p)),
               "fp_write_res")


def write_unk(path, u):
    u = np.ascontiguousarray(u, dtype=np.float64)
    nvar, n = u.shape
    _abi.check(_lib().fp_write_unk(str(path).encode(), n, nvar, u.ctypes.data_as(ctypes.c_void_p)),
               "fp_write_unk")


def read_unk(path, n, nvar=5):
    out = np.zeros((nvar, n))
    _abi.check(_lib().fp_read_unk(str(path).encode(), n, nvar, out.ctypes.data_as(ctypes.c_void_p)),
               "fp_read_unk")
    return out


def makeplot(plotreg, res_prefix, nvar, unk):
    """Merge per-domain result files <res_prefix>1.. through plotreg.reg into
    one .unk, as the reference's makeplot does."""
    _abi.check(_lib().fp_makeplot(str(plotreg).encode(), str(res_prefix).encode(), int(nvar), str(unk).encode()),
               "fp_makeplot")


def rsd_line(iteration, res1, initial_res, forces, res, force_calc_type=1):
    """One line of the .rsd residual history (writeResiduals format 504,
    mg_par:1481-1514); forces as Solver.forces() returns them, res the norms
    of Solver.residuals()."""
    f = (ctypes.c_double * 9)(*[float(x) for x in forces[:9]])
    r = (ctypes.c_double * 7)(*[float(x) for x in list(res)[:7]])
    buf = ctypes.create_string_buffer(512)
    _abi.check(_lib().fp_rsd_line(buf, len(buf), int(iteration), _c_double(res1), _c_double(initial_res), f, r,
                                  len(res), int(force_calc_type)), "fp_rsd_line")
    return buf.value.decode()


def append_rsd(path, first, iteration, res1, initial_res, forces, res, force_calc_type=1):
    """Write that line to path: a new file when first, else appended."""
    f = (ctypes.c_double * 9)(*[float(x) for x in forces[:9]])
    r = (ctypes.c_double * 7)(*[float(x) for x in list(res)[:7]])
    _abi.check(_lib().fp_append_rsd(str(path).encode(), int(bool(first)), int(iteration), _c_double(res1),
                                    _c_double(initial_res), f, r, len(res), int(force_calc_type)), "fp_append_rsd")


def cycle_line(iteration, res, maxres, scale, lift, drag):
    """The screen line of writeResiduals (format 501, mg_par:1451-1456)."""
    r = (ctypes.c_double * 5)(*[float(x) for x in res[:5]])
    m = (ctypes.c_double * 5)(*[float(x) for x in maxres[:5]])
    buf = ctypes.create_string_buffer(512)
    _abi.check(_lib().fp_cycle_line(buf, len(buf), int(iteration), r, m, _c_double(scale), _c_double(lift),
                                    _c_double(drag)), "fp_cycle_line")
    return buf.value.decode()


def primitive_to_conserved(prim):
    """The restart conversion u(2:5) = rho*u(2:5) (def_par:3850-3856)."""
    prim = np.asarray(prim, dtype=np.float64)
    u = prim.copy()
    u[1:5] = prim[0] * prim[1:5]
    return u


def splitmix64(seed, n):
    """First n outputs of the SplitMix64 generator (public-domain method by
    S. Vigna): state_i = seed + i*0x9E3779B97F4A7C15, then the mix."""
    with np.errstate(over="ignore"):
        x = np.uint64(seed) + np.arange(1, n + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)
        z = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def density_perturbation(n, seed=20261203, amplitude=0.01):
    """delta_i uniform on [-amplitude, amplitude] from SplitMix64 in file order."""
    bits = splitmix64(seed, n) >> np.uint64(11)
    u01 = bits.astype(np.float64) / float(1 << 53)
    return amplitude * (2.0 * u01 - 1.0)
