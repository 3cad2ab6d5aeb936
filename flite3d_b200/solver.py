"""Solver host mirror over the C ABI (include/flite_gpu.h).

:class:`Solver` holds one device context.  Its methods are the reference's
module calls from the multigrid driver into the grid solver
(SolverSource/mgnsg3d_mg_par.F90 into mgnsg3d_def_par.F90), one for one.
:func:`run_steady` restates the steady convergence loop of multiGridCycles
(mg_par:459-905): cycles until log10(res1/res1_first) <= -orders or
maximumnumberofcycles.

The product path is the CUDA library: constructing a Solver raises when
libflite_gpu.so is missing or no CUDA device is present; there is no CPU
fallback.
"""
import ctypes
import math

import numpy as np

from . import _abi
from .mesh import Mesh

_vp = ctypes.c_void_p


def _ptr(a):
    return a.ctypes.data_as(_vp)


def default_controls(**overrides):
    """Reference defaults (def_par:217-378) with keyword overrides applied,
    then the post-read derivation (def_par:387-415)."""
    lib = _abi.gpu_lib()
    c = _abi.Controls()
    _abi.check(lib.flite_controls_default(ctypes.byref(c)), "flite_controls_default")
    _override(c, overrides)
    _abi.check(lib.flite_controls_derive(ctypes.byref(c)), "flite_controls_derive")
    return c


def _override(c, overrides):
    """Set controls by name; an array control takes a sequence of its length."""
    for k, v in overrides.items():
        if not hasattr(c, k):
            raise KeyError(f"unknown control {k}")
        cur = getattr(c, k)
        if hasattr(cur, "__len__"):
            v = list(v)
            if len(v) != len(cur):
                raise ValueError(f"control {k} takes {len(cur)} values")
            for i, x in enumerate(v):
                cur[i] = x
        else:
            setattr(c, k, v)


def host_controls(**overrides):
    """default_controls computed by the host preprocessor library alone (the
    same defaults and derivation compiled without CUDA), for programs that
    must not load the GPU library."""
    lib = _abi.prepro_lib()
    c = _abi.Controls()
    _abi.check(lib.fp_controls_default(ctypes.byref(c)), "fp_controls_default")
    _override(c, overrides)
    _abi.check(lib.fp_controls_derive(ctypes.byref(c)), "fp_controls_derive")
    return c


def controls_from_inp(path_or_text, **overrides):
    """Defaults, then the &InputVariables deck, then overrides, then derive."""
    lib = _abi.gpu_lib()
    pre = _abi.prepro_lib()
    c = _abi.Controls()
    _abi.check(lib.flite_controls_default(ctypes.byref(c)), "flite_controls_default")
    unk = ctypes.create_string_buffer(4096)
    text = str(path_or_text)
    if "&" in text:
        rc = pre.fp_parse_inp_text(text.encode(), ctypes.byref(c), unk, len(unk))
    else:
        rc = pre.fp_read_inp(text.encode(), ctypes.byref(c), unk, len(unk))
    _abi.check(rc, "namelist read")
    _override(c, overrides)
    _abi.check(lib.flite_controls_derive(ctypes.byref(c)), "flite_controls_derive")
    return c, [u for u in unk.value.decode().split(",") if u]


class Backend:
    """A set of entry points with the flite_* signatures (the GPU library) or
    the same signatures under another prefix (the CPU checker)."""

    def __init__(self, lib, prefix):
        self.lib, self.prefix = lib, prefix

    def __getattr__(self, name):
        return getattr(self.lib, self.prefix + name)


class Solver:
    def __init__(self, controls, mesh: Mesh, backend=None):
        self.c = controls
        self.mesh = mesh
        self.be = backend or Backend(_abi.gpu_lib(), "flite_")
        self._h = _vp()
        rc = self.be.create(ctypes.byref(controls), mesh.nlevels, mesh.descs, ctypes.byref(self._h))
        if rc != _abi.FLITE_OK:
            why = self._err()
            raise RuntimeError(f"create failed with status {rc}" + (f": {why}" if why else ""))
        ng = mesh.nlevels
        if controls.numberOfGridsToUse > 0:
            ng = min(ng, controls.numberOfGridsToUse)
        self.nlevels = ng
        self.nodes = [mesh.level(l + 1).n_nodes for l in range(ng)]
        # conserved variables, plus nu~ with the Spalart-Allmaras model
        self.nvar = 6 if controls.turbulenceModel == 1 else 5

    def _err(self):
        if not hasattr(self.be.lib, self.be.prefix + "last_error"):
            return None
        buf = ctypes.create_string_buffer(1024)
        self.be.last_error(self._h, buf, len(buf))
        return buf.value.decode()

    def _ck(self, rc, what):
        if rc != _abi.FLITE_OK:
            raise RuntimeError(f"{what} failed with status {rc}: {self._err()}")

    def close(self):
        if self._h:
            self.be.destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- state -------------------------------------------------------------
    def set_state(self, u, level=1):
        u = np.ascontiguousarray(u, dtype=np.float64)
        assert u.shape == (self.nvar, self.nodes[level - 1])
        self._ck(self.be.set_state(self._h, level, _ptr(u)), "set_state")

    def get_state(self, level=1, out=None):
        u = np.zeros((self.nvar, self.nodes[level - 1])) if out is None else out
        assert u.shape == (self.nvar, self.nodes[level - 1]) and u.dtype == np.float64
        assert u.flags["C_CONTIGUOUS"]
        self._ck(self.be.get_state(self._h, level, _ptr(u)), "get_state")
        return u

    def get_pressure(self, level=1):
        p = np.zeros(self.nodes[level - 1])
        self._ck(self.be.get_pressure(self._h, level, _ptr(p)), "get_pressure")
        return p

    def init_freestream(self):
        self._ck(self.be.init_freestream(self._h), "init_freestream")

    def explicit_time_step(self):
        """ivd%physicalTimeStep after the last cycle of an explicit run (the
        smallest local time step of the last makeTimeSteps)."""
        v = ctypes.c_double()
        self._ck(self.be.explicit_time_step(self._h, ctypes.byref(v)), "explicit_time_step")
        return v.value

    def start(self):
        self._ck(self.be.start(self._h), "start")

    # ---- solver calls ------------------------------------------------------
    def next_physical_step(self):
        """Unsteady runs: close the physical time step (uold2 = uold, uold =
        u) and open the next one (viscosity reset, restrictions)."""
        self._ck(self.be.next_physical_step(self._h), "next_physical_step")

    def update_geometry(self, mesh):
        """Moving meshes (flowType 2): take the geometry the mesh now holds
        (after Mesh.set_moving) for the physical step just opened."""
        self._ck(self.be.update_geometry(self._h, mesh.nlevels, mesh.descs), "update_geometry")

    def do_time_iterations(self, level, nsteps=1, calc_diss=True, cycle=1, calc_turb=True):
        self._ck(self.be.do_time_iterations(self._h, level, nsteps, int(calc_diss), int(calc_turb), cycle),
                 "do_time_iterations")

    def restrict(self, fine_level, calc_turb=True):
        self._ck(self.be.restrict(self._h, fine_level, int(calc_turb)), "restrict")

    def prolong(self, coarse_level):
        self._ck(self.be.prolong(self._h, coarse_level), "prolong")

    def cycle(self, cycle_no):
        self._ck(self.be.cycle(self._h, cycle_no), "cycle")

    def residuals(self):
        res = (ctypes.c_double * 7)()
        mres = (ctypes.c_double * 7)()
        mind = (ctypes.c_int32 * 7)()
        rc = self.be.residuals(self._h, res, mres, mind)
        if rc == _abi.FLITE_ENAN:
            raise FloatingPointError("NaN in residual")
        self._ck(rc, "residuals")
        n = self.nvar
        return np.array(res[:n]), np.array(mres[:n]), np.array(mind[:n])

    def forces(self):
        """lift, drag, latF, frictionDrag, latM, longM, longMl, longMd, rollM
        (the last three with forceCalcType 3, else 0)."""
        out = (ctypes.c_double * 9)()
        self._ck(self.be.forces(self._h, out), "forces")
        return np.array(out[:])

    def residual_fwd(self, u, level=1):
        """makeRHS of the mean flow (5 components) at the state u of a level."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        r = np.zeros((5, u.shape[1]))
        self._ck(self.be.residual_fwd(self._h, level, _ptr(u), _ptr(r)), "residual_fwd")
        return r

    def residual_vjp(self, u, rbar, level=1):
        """ubar = (dR/du)^T rbar of residual_fwd (GPU library only)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        rbar = np.ascontiguousarray(rbar, dtype=np.float64)
        ub = np.zeros_like(u)
        self._ck(self.be.residual_vjp(self._h, level, _ptr(u), _ptr(rbar), _ptr(ub)), "residual_vjp")
        return ub

    def residual_jvp(self, u, du, level=1):
        """jv = (dR/du) du of residual_fwd (the oracle's tangent)."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        du = np.ascontiguousarray(du, dtype=np.float64)
        jv = np.zeros_like(u)
        self._ck(self.be.residual_jvp(self._h, level, _ptr(u), _ptr(du), _ptr(jv)), "residual_jvp")
        return jv

    OBJECTIVES = {"CL": 0, "CD": 1}

    def objective(self, name="CL"):
        """Lift or drag coefficient of the level-1 state with the pressure of
        the state (the objective of adjoint_solve)."""
        J = ctypes.c_double()
        self._ck(self.be.objective(self._h, self.OBJECTIVES[name], ctypes.byref(J)), "objective")
        return J.value

    def iteration_vjp(self, u, lam, geometry=False, mu=None, lam_mu=None):
        """(dG/du)^T lam of one level-1 smoother iteration G at the state u;
        with geometry=True also (dG/dg)^T lam for g = side_w, bnd_w, volume.
        In a laminar run mu is the viscosity the time step reads, lam_mu the
        adjoint of the viscosity the iteration computes, and the result ends
        with mu_bar."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        ub = np.zeros_like(u)
        d = self.mesh.level(1)
        g = [np.zeros((3, d.n_sides)), np.zeros((3, d.n_bsides)), np.zeros(d.n_nodes)] if geometry else None
        gp = [_ptr(a) for a in g] if geometry else [None, None, None]
        m = None if mu is None else np.ascontiguousarray(mu, dtype=np.float64)
        lm = None if lam_mu is None else np.ascontiguousarray(lam_mu, dtype=np.float64)
        mb = None if mu is None else np.zeros(d.n_nodes)
        self._ck(self.be.iteration_vjp(self._h, _ptr(u), _ptr(lam), _ptr(ub), *gp,
                                       *[None if a is None else _ptr(a) for a in (m, lm, mb)]), "iteration_vjp")
        out = (ub, *g) if geometry else (ub,)
        if mu is not None:
            out = out + (mb,)
        return out if len(out) > 1 else out[0]

    def iteration_jvp(self, u, du, side_w=None, bnd_w=None, volume=None, mu=None, dmu=None):
        """(G(u), dG) with dG = G_u du + G_g dg along the geometry direction
        dg = (side_w, bnd_w, volume) (None: zero) -- the oracle's tangent.  In
        a laminar run mu is the viscosity the time step reads and the result
        is (G, dG, mu', dmu') with mu' the viscosity of u."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        du = np.ascontiguousarray(du, dtype=np.float64)
        g = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (side_w, bnd_w, volume)]
        v, dv = np.zeros_like(u), np.zeros_like(u)
        m = None if mu is None else np.ascontiguousarray(mu, dtype=np.float64)
        dm = None if dmu is None else np.ascontiguousarray(dmu, dtype=np.float64)
        mo = np.zeros(u.shape[1]) if mu is not None else None
        dmo = np.zeros(u.shape[1]) if mu is not None else None
        self._ck(self.be.iteration_jvp(self._h, _ptr(u), _ptr(du), *[None if a is None else _ptr(a) for a in g],
                                       _ptr(v), _ptr(dv), *[None if a is None else _ptr(a) for a in (m, dm, mo, dmo)]),
                 "iteration_jvp")
        return (v, dv) if mu is None else (v, dv, mo, dmo)

    def objective_jvp(self, name, u, du, side_w=None, bnd_w=None, volume=None):
        """(J, dJ) of the lift or drag coefficient along (du, d side_w,
        d bnd_w, d volume) -- the oracle's tangent."""
        u = np.ascontiguousarray(u, dtype=np.float64)
        du = np.ascontiguousarray(du, dtype=np.float64)
        g = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (side_w, bnd_w, volume)]
        J, dJ = ctypes.c_double(), ctypes.c_double()
        self._ck(self.be.objective_jvp(self._h, self.OBJECTIVES[name], _ptr(u), _ptr(du),
                                       *[None if a is None else _ptr(a) for a in g], ctypes.byref(J),
                                       ctypes.byref(dJ)), "objective_jvp")
        return J.value, dJ.value

    ADJOINT_METHODS = {"fixed-point": 0, "gmres": 1}

    def set_adjoint_method(self, method="gmres", restart=50):
        """How adjoint_solve iterates: "gmres" (restarted, the default) or
        "fixed-point"."""
        self._ck(self.be.set_adjoint_method(self._h, self.ADJOINT_METHODS[method], int(restart)),
                 "set_adjoint_method")

    def adjoint_solve(self, name="CL", tol=1e-10, max_iter=100000):
        """Sensitivity of the lift or drag coefficient of the converged
        level-1 state to the level-1 geometry: dict with J, side_w_bar (3, E),
        bnd_w_bar (3, B), volume_bar (N), iterations and residual.  The
        sensitivity to node coordinates is Mesh.geometry_vjp of the three."""
        d = self.mesh.level(1)
        sw, bw, vol = np.zeros((3, d.n_sides)), np.zeros((3, d.n_bsides)), np.zeros(d.n_nodes)
        J, it, res = ctypes.c_double(), ctypes.c_int32(), ctypes.c_double()
        self._ck(self.be.adjoint_solve(self._h, self.OBJECTIVES[name], ctypes.c_double(tol), int(max_iter),
                                       ctypes.byref(J), _ptr(sw), _ptr(bw), _ptr(vol), ctypes.byref(it),
                                       ctypes.byref(res)), "adjoint_solve")
        return dict(J=J.value, side_w_bar=sw, bnd_w_bar=bw, volume_bar=vol, iterations=it.value,
                    residual=res.value)

    def set_kernel_options(self, edge_block=256, node_block=256, gather_unroll=1):
        self._ck(self.be.set_kernel_options(self._h, edge_block, node_block, gather_unroll), "set_kernel_options")

    def set_tiled_gather(self, level, mode=1):
        """How the fused central gather of a level reads its incidences: 0
        through the node's incidence list; 1..4 through the incidence rows of
        256-node blocks, with the block and its halo staged in shared memory
        (1, 2) or not (3, 4).  No effect on any result."""
        self._ck(self.be.set_tiled_gather(self._h, level, mode), "set_tiled_gather")

    def set_gather_fusion(self, level, on=1):
        """Whether a level's gathers that walk the same incidence list share
        one walk (time step with Laplacian, JST flux with viscous gradients)
        where a thread serves a node: 1 (default) or 0.  No effect on any
        result."""
        self._ck(self.be.set_gather_fusion(self._h, level, on), "set_gather_fusion")

    def set_gather_lanes(self, level, lanes):
        """Lanes per node of a level's gathers: 1, 4, 8, 16, 32 (0: default)."""
        self._ck(self.be.set_gather_lanes(self._h, level, lanes), "set_gather_lanes")

    KERNEL_GROUPS = ("pressure", "timestep", "dissipation", "visc_prim", "visc_grad", "visc_flux",
                     "flux_terms", "node_update", "ts_lap", "jflux_vgrad")

    def profile_kernels(self, level=1, reps=10):
        """{kernel group: average device ms} over one relaxation step of a level."""
        ms = (ctypes.c_double * 16)()
        n = ctypes.c_int32()
        self._ck(self.be.profile_kernels(self._h, level, reps, ms, 16, ctypes.byref(n)), "profile_kernels")
        return {k: ms[i] for i, k in enumerate(self.KERNEL_GROUPS[:n.value])}

    def profile_adjoint(self, level=1, reps=10):
        """(forward ms, adjoint ms) per residual evaluation on a level."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._ck(self.be.profile_adjoint(self._h, level, reps, ctypes.byref(a), ctypes.byref(b)),
                 "profile_adjoint")
        return a.value, b.value

    def time_cycles(self, ncycles, cycle_no=1):
        ms = ctypes.c_double()
        self._ck(self.be.time_cycles(self._h, cycle_no, ncycles, ctypes.byref(ms)), "time_cycles")
        return ms.value

    def cycle_launches(self):
        n = ctypes.c_int64()
        self._ck(self.be.cycle_launches(self._h, ctypes.byref(n)), "cycle_launches")
        return n.value

    def profile_level(self, level=1, reps=10):
        a, b = ctypes.c_double(), ctypes.c_double()
        self._ck(self.be.profile_level(self._h, level, reps, ctypes.byref(a), ctypes.byref(b)),
                 "profile_level")
        return a.value, b.value


def set_node_order(order):
    """Node numbering of the contexts created afterwards: 0 (default) the
    caller's, 1 the device's locality order.  No effect on any result; node
    arrays always cross the ABI in the caller's numbering."""
    _abi.check(_abi.gpu_lib().flite_set_node_order(int(order)), "flite_set_node_order")


def initial_state(controls, mesh, perturb_seed=None, amplitude=0.01):
    """Freestream state of level 1 as conserved variables; with a seed the
    density gets the seeded +-amplitude perturbation in primitive form (the
    velocity and E/rho stay at freestream), as a restart file would carry."""
    from .mesh import density_perturbation, primitive_to_conserved
    n = mesh.level(1).n_nodes
    inf = list(controls.inflowField)
    prim = np.empty((5, n))
    for k in range(5):
        prim[k] = inf[k]
    prim[0] = inf[0]
    if perturb_seed is not None:
        prim[0] = inf[0] * (1.0 + density_perturbation(n, perturb_seed, amplitude))
    u = primitive_to_conserved(prim)
    if controls.turbulenceModel == 1:
        # nu~ of the freestream initialisation (def_par:3961-3963)
        u = np.vstack([u, np.full((1, n), 0.1)])
    return u


def run_steady(solver, orders=8.0, max_cycles=1000, callback=None, rsd=None, screen=None):
    """Convergence loop of multiGridCycles (mg_par:789-816): cycles until
    log(res0)-log(res) >= orders*log(10) or max_cycles.  Returns the history
    of (cycle, res1, lift, drag).  With rsd (a path) every cycle appends the
    residual-history line of writeResiduals to that file, the first cycle
    starting it afresh; with screen (a callable taking a string) every cycle
    passes it the reference's screen line (mg_par:1449-1516)."""
    from .mesh import append_rsd, cycle_line
    hist = []
    res0 = None
    for it in range(1, max_cycles + 1):
        solver.cycle(it)
        res, maxres, _ = solver.residuals()
        f = solver.forces()
        if res0 is None:
            res0 = res[0]
        hist.append((it, res[0], f[0], f[1]))
        if rsd is not None:
            append_rsd(rsd, it == 1, it, res[0], res0, f, res, solver.c.forceCalcType)
        if screen is not None:
            scale = 1.0 / float(solver.c.numberOfProcesses * solver.nodes[0])
            screen(cycle_line(it, res[:5], maxres[:5], scale, f[0], f[1]))
        if callback:
            callback(it, res, f)
        if not (math.log(res0) - math.log(res[0]) < math.log(10.0) * orders):
            break
    return hist


def run_unsteady(solver, steps, cycles_per_step, callback=None):
    """Dual time stepping of multiGridCycles for flowType 1 (mg_par:483-890):
    per physical step a fixed number of multigrid cycles (numberOfMGIterations
    > 0), then the step is closed and the next one opened.  Returns the
    (step, res1, lift, drag) at the end of each step."""
    hist = []
    for step in range(1, steps + 1):
        for it in range(1, cycles_per_step + 1):
            solver.cycle(it)
        res, _, _ = solver.residuals()
        f = solver.forces()
        hist.append((step, res[0], f[0], f[1]))
        if callback:
            callback(step, res, f)
        if step < steps:
            solver.next_physical_step()
    return hist


class Batch:
    """Many solves (mesh x flow condition) advanced together: one CUDA-graph
    launch per batch cycle; cases on one mesh share the mesh's device copy
    and, where their controls take the same kernels, every launch of the
    cycle (a case group)."""

    def __init__(self, cases):
        """cases: list of (controls, mesh) pairs."""
        lib = _abi.gpu_lib()
        self._lib = lib
        meshes, mesh_of = [], []
        for _, m in cases:
            for k, mm in enumerate(meshes):
                if mm is m:
                    mesh_of.append(k)
                    break
            else:
                meshes.append(m)
                mesh_of.append(len(meshes) - 1)
        self.meshes = meshes
        n = len(cases)
        ctl = (_abi.Controls * n)(*[c for c, _ in cases])
        mof = (ctypes.c_int32 * n)(*mesh_of)
        nlev = (ctypes.c_int32 * len(meshes))(*[m.nlevels for m in meshes])
        lv = (ctypes.c_void_p * len(meshes))(*[ctypes.addressof(m.descs) for m in meshes])
        self._h = _vp()
        rc = lib.flite_batch_create(n, ctl, mof, len(meshes), nlev, lv, ctypes.byref(self._h))
        if rc != _abi.FLITE_OK:
            raise RuntimeError(f"flite_batch_create failed with status {rc}")
        self.cases = []
        for i, (c, m) in enumerate(cases):
            h = _vp()
            _abi.check(lib.flite_batch_context(self._h, i, ctypes.byref(h)), "flite_batch_context")
            s = Solver.__new__(Solver)
            s.c, s.mesh, s.be, s._h = c, m, Backend(lib, "flite_"), h
            ng = m.nlevels if c.numberOfGridsToUse <= 0 else min(m.nlevels, c.numberOfGridsToUse)
            s.nlevels = ng
            s.nodes = [m.level(l + 1).n_nodes for l in range(ng)]
            s.nvar = 6 if c.turbulenceModel == 1 else 5
            s.close = lambda: None  # owned by the batch
            self.cases.append(s)

    def cycle(self, cycle_no):
        _abi.check(self._lib.flite_batch_cycle(self._h, cycle_no), "flite_batch_cycle")

    def run(self, orders=8.0, max_cycles=1000, first_cycle=1, check_every=1):
        """Cycle every case until its res1 falls by 10^-orders (or max_cycles);
        returns (cycles run per case, log10 residual reduction per case)."""
        n = len(self.cases)
        cyc = (ctypes.c_int32 * n)()
        red = (ctypes.c_double * n)()
        _abi.check(self._lib.flite_batch_run(self._h, first_cycle, max_cycles, ctypes.c_double(orders),
                                             check_every, cyc, red), "flite_batch_run")
        return np.array(cyc[:]), np.array(red[:])

    def time_cycles(self, ncycles, cycle_no=1, sequential=False):
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        _abi.check(self._lib.flite_batch_time_cycles(self._h, cycle_no, ncycles, int(sequential),
                                                     ctypes.byref(ms), ctypes.byref(n)),
                   "flite_batch_time_cycles")
        return ms.value, n.value

    def autotune(self, reps=3, cycle_no=1):
        e, n, ms = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
        _abi.check(self._lib.flite_batch_autotune(self._h, cycle_no, reps, ctypes.byref(e),
                                                  ctypes.byref(n), ctypes.byref(ms)),
                   "flite_batch_autotune")
        return e.value, n.value, ms.value

    def set_blocks(self, edge_block, node_block):
        _abi.check(self._lib.flite_batch_set_blocks(self._h, edge_block, node_block),
                   "flite_batch_set_blocks")

    def autotune_lanes(self, reps=2, cycle_no=1, nlevels=8):
        """Lanes per node of each level's gathers, timed level by level
        (coarsest first) and set on every case; returns the choice per level
        and the best batch-cycle time in ms."""
        lanes = (ctypes.c_int32 * nlevels)()
        ms = ctypes.c_double()
        _abi.check(self._lib.flite_batch_autotune_lanes(self._h, cycle_no, reps, nlevels, lanes, ctypes.byref(ms)),
                   "flite_batch_autotune_lanes")
        return [v for v in lanes[:] if v], ms.value

    def set_grouping(self, on):
        """Case groups on (the default) or off: with them every kernel of the
        cycle runs once for all the cases on one mesh."""
        _abi.check(self._lib.flite_batch_set_grouping(self._h, int(bool(on))), "flite_batch_set_grouping")

    def grouping(self):
        """Whether case groups are on (the autotuner keeps the faster mode)."""
        n = ctypes.c_int32()
        _abi.check(self._lib.flite_batch_grouping(self._h, ctypes.byref(n)), "flite_batch_grouping")
        return bool(n.value)

    def groups(self):
        """The case groups of the last batch graph."""
        n = ctypes.c_int32()
        _abi.check(self._lib.flite_batch_groups(self._h, ctypes.byref(n)), "flite_batch_groups")
        return n.value

    def close(self):
        if self._h:
            self._lib.flite_batch_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
