"""Benchmark of the B200 flow-solver hot path: multigrid cycles per second.

One step is one multigrid cycle (oneCycle, SolverSource/mgnsg3d_mg_par.F90:
907-1196) of the growing V-cycle over every level, on the bump-channel mesh
264x88x88 hexes split into tets (2,099,065 nodes, 14,473,976 edges, 4
agglomerated levels), seeded synthetic initial state.  The mesh and state
far exceed the 126 MB L2, so no flush is needed between timed cycles.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 (one process per GPU under torchrun) every rank runs an
independent replica of the solve: the path does not shard (one mesh per GPU,
no collectives on the data path); value = cycles of all ranks / max time.
--impl reference times the CPU restatement of the reference solver (the
Fortran reference cannot be compiled here) on the host cores instead.
"""
import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

MESH = dict(nx=264, ny=88, nz=88, bump=0.05, levels=4)
METRIC = "MG cycles/s"
CONTROLS = dict(ReynoldsNumber=5000.0, MachNumber=0.5, alpha=0.0, CFLNumber=2.0, fluxType=1,
                multigridScheme=3, numberOfGridsToUse=4, wallsAreIsentropic=1, viscosityScheme=1)
def workload(nodes=None, edges=None):
    """The workload's name, with the mesh's size (the default mesh's when not given)."""
    nodes = 2099065 if nodes is None else nodes
    edges = 14473976 if edges is None else edges
    return ("laminar Navier-Stokes, Re 5e3, M 0.5, adiabatic walls, on the bump channel "
            f"{MESH['nx']}x{MESH['ny']}x{MESH['nz']} hex -> 6 tets ({nodes:,} nodes, {edges:,} edges), "
            f"{MESH['levels']} agglomerated MG levels, growing V-cycle, 3-stage RK, CFL 2, central flux + JST, FP64")


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4)
                          if len(s) > 5 + k and s[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def build_case(host_only=False):
    """The mesh, controls and seeded initial state of the workload.  With
    host_only the controls come from the host preprocessor library, so the
    CUDA library is never loaded (the CPU reference arm)."""
    import flite3d_b200 as F
    t0 = time.time()
    mesh = F.Mesh.bump_channel(MESH["nx"], MESH["ny"], MESH["nz"], MESH["bump"], MESH["levels"])
    c = F.host_controls(**CONTROLS) if host_only else F.default_controls(**CONTROLS)
    u0 = F.initial_state(c, mesh, perturb_seed=20261203, amplitude=0.01)
    return F, mesh, c, u0, time.time() - t0


def apply_options(solver, options, unroll=1):
    """Set the tuned launch options (node block, lanes, incidence-row mode
    and shared walks per level) on a solver; none changes a result."""
    if not options:
        return
    solver.set_kernel_options(256, options["node_block"], unroll)
    for lvl, g in options["lanes"].items():
        solver.set_gather_lanes(lvl, g)
        solver.set_tiled_gather(lvl, options["tiled"][lvl] if g == 1 else 0)
        solver.set_gather_fusion(lvl, options["fuse"][lvl])


def node_kernel_name(lanes, tiled, unroll):
    """The instance of the level-1 node kernel the tuned launch options run."""
    what = ("(level 1: central fluxes of the incident edges computed in the node gather, fused with the RK "
            "stage update")
    if lanes == 1 and tiled:
        minb, stage = (2, True) if tiled == 1 else (3, True) if tiled == 2 else (2, False) if tiled == 3 else (3, False)
        return (f"k_node_update_tiled<{minb}, {str(stage).lower()}> {what}; incidences read through the incidence "
                "rows of 256-node blocks" + (", blocks and halo staged in shared memory)" if stage else ")"))
    if lanes == 1 and unroll == 2:
        return f"k_node_update<GATHER_CENTRAL2, 1> {what})"
    if lanes == 1:  # the bench workload has no engines and no explicit stepping
        return f"k_node_update<GATHER_LEAN, 1> {what}; node tail without the engine and explicit branches)"
    return f"k_node_update<GATHER_CENTRAL, {lanes}> {what})"


def node_kernel_bytes(mesh):
    """Algorithmic bytes of one launch of the dominant kernel on level 1: the
    node kernel that computes the central fluxes of every incident edge and
    applies the RK stage update (measured in restrictGrid's fine-increment
    mode, which has the stage's read set).  Per node: the 48-byte state
    record (own and neighbours' reads of one array, counted once), uprev
    (40 B), dissipation (40 B), dt and volume (16 B), u(rho) (8 B), boundary
    class (1 B), two CSR offsets (8 B) and the result (40 B); per interior
    edge its two 8-byte incidence entries and its 32-byte coefficient record;
    per boundary edge two incidence entries and two 40-byte contributions; per
    boundary node its normal (24 B)."""
    d = mesh.level(1)
    return d.n_nodes * (48 + 40 + 40 + 16 + 8 + 1 + 8 + 40) + d.n_sides * 48 + d.n_bsides * 88 \
        + d.n_bnodes * 24


def group_bytes(mesh, dissipation_weighting=False):
    """Algorithmic bytes of each level-1 kernel group of one relaxation step
    (the groups of flite_profile_kernels, laminar FP64 with the scalar JST and
    a thread per node).  Every array is counted once per launch (a node's own
    and its neighbours' reads of an array are one read), an incidence entry
    is 8 bytes (two per interior edge), a boundary incidence 4 (two per
    boundary edge), a CSR offset 4 per node and list:
      pressure   u (40) in, p (8) and the 48-byte central-flux record out;
      timestep   u0..3 (32), p, mu, volume (24), two offsets (8), dt and V/dt
                 out (16); per edge two incidences and wx, wy, wz (24); per
                 boundary edge its two incidences, node pair (8) and
                 coefficients (24);
      dissipation (k_jst_lap + k_jst_flux) u (40), p, connectivity, sensor
                 out and in (8 each), the Laplacian out and in (40 each), V/dt
                 (8), dissipation out (40), two offsets; per edge its two
                 incidences twice (and the edge length twice with dissipation
                 weighting);
      visc_prim  u0..3 and p in (40), u, v, w, T out (32);
      visc_grad  u, v, w, T (32), volume, p, rho (24), class (1), offsets (8),
                 mu (8) and tau (72) out; per edge two incidences and its
                 coefficients (40); per boundary edge as in timestep (40);
                 per boundary node its normal (24) and wall stress out (24);
      visc_flux  tau (72), u, v, w (24), dissipation 1..4 in and out (64),
                 offsets (8); per edge 40; per boundary edge 40 and its code (4);
      node_update as node_kernel_bytes;
      ts_lap     (the shared walk of timestep and the Laplacian) u (40), p, mu,
                 volume, connectivity (32), offsets (8), dt and V/dt out (16),
                 Laplacian and sensor out (48); per edge and boundary edge as
                 in timestep;
      jflux_vgrad (the shared walk of the JST flux and visc_grad) Laplacian,
                 u (80), V/dt, connectivity, sensor (24), dissipation out
                 (40), u, v, w, T (32), volume, p (16), class (1), offsets
                 (8), mu and tau out (80); per edge, boundary edge and boundary
                 node as in visc_grad.
    With shared walks the timestep, dissipation and visc_grad groups launch
    nothing (the viscous workload) and are left out of the fractions."""
    d = mesh.level(1)
    N, E, B, Nb = d.n_nodes, d.n_sides, d.n_bsides, d.n_bnodes
    return {
        "pressure": N * (40 + 8 + 48),
        "timestep": N * (32 + 8 + 8 + 8 + 8 + 16) + E * (16 + 24) + B * (8 + 8 + 24),
        "dissipation": N * (40 + 8 + 8 + 8 + 8 + 40 + 40 + 8 + 40 + 8) + E * 32
        + (E * 16 if dissipation_weighting else 0),
        "visc_prim": N * (40 + 32),
        "visc_grad": N * (32 + 24 + 1 + 8 + 8 + 72) + E * 40 + B * 40 + Nb * 48,
        "visc_flux": N * (72 + 24 + 64 + 8) + E * 40 + B * 44,
        "node_update": node_kernel_bytes(mesh),
        # the shared walks: the two groups' bytes less what the second walk
        # would read again (incidences, offsets, edge coefficients and the
        # arrays both read)
        "ts_lap": N * (40 + 8 + 8 + 8 + 8 + 8 + 16 + 40 + 8) + E * (16 + 24) + B * (8 + 8 + 24),
        "jflux_vgrad": N * (40 + 40 + 8 + 8 + 8 + 40 + 32 + 8 + 8 + 1 + 8 + 8 + 72) + E * (16 + 24) + B * 40
        + Nb * 48,
    }


def group_roofline(ms, nbytes, hbm):
    """{group: {ms, algorithmic_bytes, achieved GB/s, frac}} of the groups
    that have a byte count."""
    out = {}
    for k, b in nbytes.items():
        if k in ms and ms[k] > 0:
            gbs = b / (ms[k] / 1e3) / 1e9
            out[k] = {"ms": ms[k], "algorithmic_bytes": b, "achieved_gbs": gbs, "frac": gbs / hbm}
    return out


# DRAM traffic of the dominant kernel per algorithmic byte, from an ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum) of one launch on the
# 192x64x64 bump channel (453.8 MB measured against 448.8 MB algorithmic,
# the lean node tail); the bench mesh is too large to capture with --set
# full, and the traffic scales with the nodes and edges processed
NCU_TRAFFIC_PER_ALGORITHMIC_BYTE = (425.17888 + 28.584448) / 448.800825


def run_ours(args):
    ws, rank, local = _dist()
    import torch
    import torch.distributed as dist
    if not torch.cuda.is_available():
        raise SystemExit("no CUDA device: the product path has no CPU fallback")
    torch.cuda.set_device(local)
    if ws > 1:
        dist.init_process_group("nccl", init_method="env://",
                                timeout=__import__("datetime").timedelta(seconds=600))
    from flite3d_b200 import replicas
    F, mesh, c, u0, t_mesh = build_case()
    F.solver.set_node_order(args.node_order)
    solver = F.Solver(c, mesh)
    solver.set_state(u0)
    solver.start()
    # pick the launch options on this GPU (none changes a result): node-kernel
    # block size and gather unroll by the level-1 node kernel, then the level
    # size below which gathers use a warp per node by the time of whole cycles
    tuning = {}
    if args.kernel_options:
        # fixed options (profiling runs: no tuning launches before the cycles)
        v = [int(x) for x in args.kernel_options.split(",")]
        best = (v[0], v[1])
        lanes = {lvl: v[1 + lvl] for lvl in range(1, solver.nlevels + 1)}
        tm = [int(x) for x in args.tiled_modes.split(",")] if args.tiled_modes else []
        tiled = {lvl: (tm[lvl - 1] if lvl - 1 < len(tm) else 1) for lvl in range(1, solver.nlevels + 1)}
        fz = [int(x) for x in args.fusion.split(",")] if args.fusion else []
        fuse = {lvl: (fz[lvl - 1] if lvl - 1 < len(fz) else 1) for lvl in range(1, solver.nlevels + 1)}
    else:
        for nb in (128, 256):
            for unroll in (1, 2):
                solver.set_kernel_options(256, nb, unroll)
                tuning[(nb, unroll)] = solver.profile_level(1, reps=5)[1]
        best = min(tuning, key=tuning.get)
    solver.set_kernel_options(256, best[0], best[1])
    # lanes per node of each level's gathers (and, with a thread per node,
    # whether the fused central gather stages node blocks in shared memory:
    # through the incidence rows of node blocks: modes 1..4, 0 off), by the
    # device time of that level's kernels over one relaxation step
    # (and, with the incidence lists, whether gathers that walk the same list
    # share one walk), by the device time of that level's kernels over one
    # relaxation step
    tuning_levels = {}
    if not args.kernel_options:
        lanes, tiled, fuse = {}, {}, {}
        for lvl in range(1, solver.nlevels + 1):
            t = {}
            for g in ((1, 4, 8) if lvl == 1 else (1, 4, 8, 16, 32)):
                solver.set_gather_lanes(lvl, g)
                for mode in ((0, 1, 2, 3, 4) if g == 1 else (0,)):
                    solver.set_tiled_gather(lvl, mode)
                    for fz in ((1, 0) if g == 1 and mode == 0 else (1,)):
                        solver.set_gather_fusion(lvl, fz)
                        groups = solver.profile_kernels(lvl, reps=5)
                        t[(g, mode, fz)] = sum(groups.values())
                        if lvl <= 2 and g == 1:
                            key = f"{lvl}_groups_tiled{mode}" + (("_shared" if fz else "_separate") if mode == 0 else "")
                            tuning_levels[key] = groups
            lanes[lvl], tiled[lvl], fuse[lvl] = min(t, key=t.get)
            tuning_levels[lvl] = {f"lanes{g}_tiled{m}" + (f"_shared{f}" if g == 1 and m == 0 else ""): v
                                  for (g, m, f), v in t.items()}
    options = {"node_block": best[0], "lanes": lanes, "tiled": tiled, "fuse": fuse}
    apply_options(solver, options, best[1])
    solver.set_state(u0)
    solver.start()
    # warm-up (also captures the cycle graph)
    for i in range(1, args.warmup + 1):
        solver.cycle(i)
    res, _, _ = solver.residuals()
    launches_per_cycle = solver.cycle_launches()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms = solver.time_cycles(args.steps, cycle_no=args.warmup + 1)
    torch.cuda.synchronize()
    value, ms_max = replicas.replica_rate(ms, args.steps)

    # kernel-level timing of the dominant kernel on level 1
    _, node_ms = solver.profile_level(1, reps=20)
    # adjoint cost ratio: one adjoint product against one forward residual
    # evaluation on level 1 (same level, FP64)
    fwd_ms, vjp_ms = solver.profile_adjoint(1, reps=20)
    # device ms of the kernel groups of one level-1 relaxation step
    kernels_l1 = solver.profile_kernels(1, reps=10)
    kernels_coarse = {f"level{l}": solver.profile_kernels(l, reps=10) for l in range(2, solver.nlevels + 1)}
    hbm, peak_kind = _peaks()
    nbytes = node_kernel_bytes(mesh)
    achieved = nbytes / (node_ms / 1e3) / 1e9

    # end to end through the public API with host buffers: per cycle the
    # level-1 state goes host->device from pinned memory, the cycle runs, and
    # the residual norms, forces and state come back to the host
    n = mesh.level(1).n_nodes
    pin = torch.empty((5, n), dtype=torch.float64, pin_memory=True)
    host_u = pin.numpy()
    solver.get_state(1, out=host_u)
    cyc = args.warmup + args.steps + 1
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(args.steps):
        solver.set_state(host_u)
        solver.cycle(cyc + k)
        r, _, _ = solver.residuals()
        fc = solver.forces()
        solver.get_state(1, out=host_u)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    # the resident variant: per cycle only the cycle number goes in and the
    # residual norms and forces come out (the state stays on the device, as
    # when the whole multigrid loop is driven through the library)
    t1 = time.perf_counter()
    for k in range(args.steps):
        solver.cycle(cyc + args.steps + k)
        r, _, _ = solver.residuals()
        fc = solver.forces()
    torch.cuda.synchronize()
    resident_s = time.perf_counter() - t1
    e2e_value = ws * args.steps / replicas.max_over_ranks(e2e_s)

    # the same workload with FLITE_MIXED (FP32 flux increments over an FP64
    # anchor): cycles per second
    mixed = None
    if not args.no_mixed:
        solver_m = F.Solver(F.default_controls(**CONTROLS, precision=1), mesh)
        apply_options(solver_m, options)
        solver_m.set_state(u0)
        solver_m.start()
        for i in range(1, args.warmup + 1):
            solver_m.cycle(i)
        torch.cuda.synchronize()
        ms_m = solver_m.time_cycles(args.steps, cycle_no=args.warmup + 1)
        delta_ms, node_m_ms = solver_m.profile_level(1, reps=20)
        solver_m.close()
        v_m, ms_m = replicas.replica_rate(ms_m, args.steps)
        mixed = {"value": v_m, "unit": "cycles/s", "ms_per_step": ms_m / args.steps,
                 "node_kernel_ms": node_m_ms, "increment_records_ms": delta_ms}
    ttc = None
    if not args.no_converge:
        ttc = time_to_converge(F, mesh, c, u0, args.converge_max, options)

    cpu = None
    parity = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(mesh, c, u0, cycles=args.cpu_cycles)
    if rank == 0 and ws == 1 and args.parity_cycles > 0:
        parity = parity_check(F, mesh, c, u0, args.parity_cycles, options)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "cycles/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (generated bump-channel mesh, seeded +-1% density perturbation)",
        "config": {"workload": workload(mesh.level(1).n_nodes, mesh.level(1).n_sides),
                   "mesh_nodes": mesh.level(1).n_nodes,
                   "mesh_edges": mesh.level(1).n_sides, "levels": mesh.nlevels,
                   "parallelism": f"replicas{ws}" if ws > 1 else "single",
                   "l2": "inputs larger than L2 (state+mesh+edge buffer > 1 GB)",
                   "mesh_build_s": round(t_mesh, 2)},
        "e2e": {"value": e2e_value, "unit": "cycles/s", "h2d_bytes_per_step": 5 * n * 8 + 4,
                "d2h_bytes_per_step": 5 * n * 8 + 15 * 8 + 9 * 8,
                "what": "per cycle: level-1 state host->device from pinned memory, flite_cycle, "
                        "residual norms and forces read back, level-1 state device->host",
                "resident": {"value": args.steps / resident_s, "h2d_bytes_per_step": 4,
                             "d2h_bytes_per_step": 15 * 8 + 9 * 8}},
        "gpu_launches": int(launches_per_cycle * args.steps),
        "roofline": {"kernel": node_kernel_name(lanes[1], tiled[1], best[1]),
                     "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": peak_kind,
                     "algorithmic_bytes": nbytes, "launch_ms": node_ms,
                     "traffic": nbytes * NCU_TRAFFIC_PER_ALGORITHMIC_BYTE,
                     "traffic_source": "ncu capture of one launch on the 192x64x64 mesh, "
                                       "scaled by the units processed"},
        "clocks": clk.summary(),
        "node_order": args.node_order,
        "residual_after_warmup": float(res[0]),
        "level1_kernel_ms": kernels_l1,
        "level1_roofline": group_roofline(kernels_l1, group_bytes(mesh), hbm),
        "coarse_kernel_ms": kernels_coarse,
        "node_kernel_options": {"chosen": {"node_block": best[0], "gather_unroll": best[1],
                                           "gather_lanes_per_level": lanes, "tiled_mode_per_level": tiled,
                                           "shared_walks_per_level": fuse},
                                "ms": {f"nb{k[0]}_unroll{k[1]}": v for k, v in tuning.items()},
                                "level_ms": tuning_levels},
        "adjoint": {"fwd_ms": fwd_ms, "vjp_ms": vjp_ms, "cost_ratio": vjp_ms / fwd_ms,
                    "what": "flite_residual_vjp vs flite_residual_fwd kernels on level 1, FP64"},
    }
    if mixed is not None:
        line["mixed"] = mixed
    if ttc is not None:
        line["time_to_1e-8"] = ttc
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if parity is not None:
        line["parity"] = parity
    print(json.dumps(line), flush=True)


def time_to_converge(F, mesh, c, u0, max_cycles, options=None):
    """Wall time from the first cycle until res1 <= 1e-8 res1(cycle 1), for
    FP64 and FLITE_MIXED on the same workload, with lift and drag there."""
    import torch
    out = {}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        cc = F.default_controls(**CONTROLS, precision=prec)
        s = F.Solver(cc, mesh)
        apply_options(s, options)
        s.set_state(u0)
        s.start()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r0 = None
        cyc = 0
        for cyc in range(1, max_cycles + 1):
            s.cycle(cyc)
            r = s.residuals()[0][0]
            r0 = r0 or r
            if r <= 1e-8 * r0:
                break
        secs = time.perf_counter() - t0
        f = s.forces()
        out[name] = {"seconds": secs, "cycles": cyc, "reached": bool(r <= 1e-8 * r0),
                     "log10_reduction": float(math.log10(r / r0)), "CL": float(f[0]), "CD": float(f[1])}
        s.close()
    a, b = out["fp64"], out["mixed"]
    if a["reached"] and b["reached"]:
        out["speedup_mixed"] = a["seconds"] / b["seconds"]
        out["CL_rel_diff"] = abs(b["CL"] - a["CL"]) / max(abs(a["CL"]), 1e-300)
        out["CD_rel_diff"] = abs(b["CD"] - a["CD"]) / max(abs(a["CD"]), 1e-300)
    return out


def parity_check(F, mesh, c, u0, cycles, options=None):
    """The bench workload itself, GPU against the CPU restatement: both
    start from the seeded state u0 and run the same `cycles` growing-V
    cycles (the restatement single-threaded, in the reference's edge order);
    then every level's state is compared bit for bit, and the residual norms
    and forces, which the GPU sums in another order, relatively."""
    import torch
    from flite3d_b200.solver import Backend, Solver
    import flite3d_b200.build as b
    b.build_oracle()
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_build", "liboracle.so"))
    lib.oracle_set_threads(1)
    g = F.Solver(c, mesh)
    apply_options(g, options)
    o = Solver(c, mesh, backend=Backend(lib, "oracle_"))
    t0 = time.perf_counter()
    for s in (g, o):
        s.set_state(u0)
        s.start()
        for cyc in range(1, cycles + 1):
            s.cycle(cyc)
    torch.cuda.synchronize()
    levels = []
    for level in range(1, g.nlevels + 1):
        a, r = g.get_state(level), o.get_state(level)
        levels.append({"level": level, "nodes": int(a.shape[1]), "bitwise": bool(np.array_equal(a, r)),
                       "max_abs": float(np.abs(a - r).max())})
    rg, ro = g.residuals()[0], o.residuals()[0]
    fg, fo = g.forces(), o.forces()
    g.close()
    o.close()
    return {"cycles": cycles, "bitwise": all(x["bitwise"] for x in levels),
            "max_abs": max(x["max_abs"] for x in levels), "levels": levels,
            "residual_max_rel": float(np.max(np.abs(rg - ro) / np.abs(ro))),
            "CL_rel": float(abs(fg[0] - fo[0]) / abs(fo[0])), "CD_rel": float(abs(fg[1] - fo[1]) / abs(fo[1])),
            "seconds": time.perf_counter() - t0,
            "what": f"GPU vs the single-threaded CPU restatement from the same seeded state, {cycles} cycles of "
                    "the bench workload; states compared with np.array_equal on every level"}


def cpu_baseline(mesh, c, u0, cycles=2, sample_of="the same 2.1M-node workload"):
    """The CPU restatement (oracle/) timed on the host: a bounded sample of the
    same workload (a few cycles of the same mesh and controls)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import flite3d_b200.build as b
    from flite3d_b200.solver import Backend, Solver
    b.build_oracle()
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_build", "liboracle.so"))
    threads = host_threads()
    lib.oracle_set_threads(threads)
    o = Solver(c, mesh, backend=Backend(lib, "oracle_"))
    o.set_state(u0)
    o.start()
    o.cycle(1)  # warm the caches
    t0 = time.perf_counter()
    for i in range(cycles):
        o.cycle(2 + i)
    dt = time.perf_counter() - t0
    # the same restatement on one thread (the reference's loop order)
    lib.oracle_set_threads(1)
    t1 = time.perf_counter()
    o.cycle(2 + cycles)
    dt1 = time.perf_counter() - t1
    lib.oracle_set_threads(threads)
    o.close()
    return {"value": cycles / dt, "unit": "cycles/s", "cores": threads, "kind": "port",
            "single_thread": {"value": 1.0 / dt1, "cycles": 1},
            "sample": f"{cycles} cycles of {sample_of} after one warm-up cycle, "
                      f"FP64 C++ restatement on {threads} threads (edge loops over coloured "
                      "blocks of edges)"}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference(args):
    ws, rank, local = _dist()
    if rank != 0:
        return
    F, mesh, c, u0, _ = build_case(host_only=True)
    import flite3d_b200.build as b
    from flite3d_b200.solver import Backend, Solver
    b.build_oracle()
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_build", "liboracle.so"))
    threads = host_threads()
    lib.oracle_set_threads(threads)
    o = Solver(c, mesh, backend=Backend(lib, "oracle_"))
    o.set_state(u0)
    o.start()
    # the requested warm-up, at most 3 cycles, and a bounded sample of the
    # timed cycles (about a second each on the 2.1M-node mesh)
    warm = max(1, min(args.warmup, 3))
    for i in range(1, warm + 1):
        o.cycle(i)
    steps = max(1, min(args.steps, args.cpu_cycles))
    t0 = time.perf_counter()
    for i in range(steps):
        o.cycle(warm + 1 + i)
    dt = time.perf_counter() - t0
    v = steps / dt
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "cycles/s", "n_gpus": 0,
        "steps": steps, "warmup": warm, "ms_per_step": dt / steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload(mesh.level(1).n_nodes, mesh.level(1).n_sides)},
        "requested": {"steps": args.steps, "warmup": args.warmup,
                      "why_fewer": "a bounded CPU sample: each cycle of the 2.1M-node workload takes about "
                                   "a second on the host, so at most --cpu-cycles timed cycles after at most "
                                   "3 warm-up cycles"},
        "cpu_baseline": {"value": v, "unit": "cycles/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} cycles after {warm} warm-up cycles on {threads} threads; the "
                                   "Fortran reference cannot be compiled here (no Fortran "
                                   "compiler), so the CPU restatement of it runs"},
        "e2e": {"value": v, "unit": "cycles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def run_rans(args):
    """The RANS configuration: Spalart-Allmaras on the extruded
    NACA0012 O-grid (200 x 120 x 240 cells: 40 wall layers from 1e-5 chord
    growing by 1.15, far field at 20 chords, one chord of span), Re 6e6,
    M 0.8, alpha 1.25, HLLC order 2 with Galerkin gradients, 5 levels, FP64.
    One JSON line: MG cycles/s (device time of graph-replayed cycles)."""
    import torch
    import flite3d_b200 as F
    if not torch.cuda.is_available():
        raise SystemExit("no CUDA device: the product path has no CPU fallback")
    t0 = time.time()
    mesh = F.Mesh.naca0012(args.rans_ni, args.rans_nj, args.rans_nk, first_cell=1.0e-5, growth=1.15, nlayer=40,
                           farfield=20.0, span=1.0, nlevels=5)
    t_mesh = time.time() - t0
    c = F.default_controls(ReynoldsNumber=6.0e6, MachNumber=0.8, alpha=1.25, CFLNumber=1.0, fluxType=4,
                           HLLCFluxOrder=2, Automaticlipping=1, GradientMethod=1, multigridScheme=3,
                           numberOfGridsToUse=5, turbulenceModel=1, wallsAreIsentropic=1)
    F.solver.set_node_order(args.node_order)
    s = F.Solver(c, mesh)
    s.init_freestream()
    s.start()
    for i in range(1, args.warmup + 1):
        s.cycle(i)
    torch.cuda.synchronize()
    ms = s.time_cycles(args.steps, cycle_no=args.warmup + 1)
    res = s.residuals()[0]
    d = mesh.level(1)
    print(json.dumps({
        "metric": METRIC, "value": args.steps / (ms / 1e3), "unit": "cycles/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (generated NACA0012 O-grid, freestream start)",
        "config": {"workload": "RANS Spalart-Allmaras, Re 6e6, M 0.8, alpha 1.25, HLLC order 2, on the extruded "
                               f"NACA0012 O-grid {args.rans_ni}x{args.rans_nj}x{args.rans_nk} hex -> 6 tets, "
                               "5 agglomerated MG levels, growing V-cycle",
                   "mesh_nodes": d.n_nodes, "mesh_edges": d.n_sides, "levels": mesh.nlevels,
                   "mesh_build_s": round(t_mesh, 2)},
        "residuals_after": [float(x) for x in res], "gpu_launches": s.cycle_launches() * args.steps,
        "node_order": args.node_order,
    }), flush=True)


UPWIND = dict(ReynoldsNumber=0.0, MachNumber=0.5, alpha=0.0, CFLNumber=2.0, fluxType=3, reconstruction=1,
              rungeKuttaStages=5, secondOrderDissipationFactor=0.0, fourthOrderDissipationFactor=0.0,
              multigridScheme=3, numberOfGridsToUse=3)


def run_upwind(args):
    """The bump-channel Euler case with the upwind extension (no reference
    counterpart): Roe flux with MUSCL reconstruction from the Galerkin
    gradients and the Van Albada limiter on level 1, five stages
    (1/4, 1/6, 3/8, 1/2, 1), CFL 2, M 0.5, 3 agglomerated levels, seeded
    +-1% density start.  One JSON line: MG cycles/s (device time of
    graph-replayed cycles), the wall time to an 8-order residual drop, and
    the CPU restatement of the same extension timed on the host."""
    import torch
    import flite3d_b200 as F
    if not torch.cuda.is_available():
        raise SystemExit("no CUDA device: the product path has no CPU fallback")
    nx, ny, nz = [int(v) for v in args.upwind_mesh.split(",")]
    mesh = F.Mesh.bump_channel(nx, ny, nz, 0.05, nlevels=3)
    c = F.default_controls(**UPWIND)
    u0 = F.initial_state(c, mesh, perturb_seed=20261203, amplitude=0.01)
    s = F.Solver(c, mesh)
    s.set_state(u0)
    s.start()
    for i in range(1, args.warmup + 1):
        s.cycle(i)
    torch.cuda.synchronize()
    ms = s.time_cycles(args.steps, cycle_no=args.warmup + 1)
    launches = s.cycle_launches() * args.steps
    s.close()
    # time to converge: res1 down 8 orders (numberOfMGIterations = -8)
    s = F.Solver(c, mesh)
    s.set_state(u0)
    s.start()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r0 = r = None
    cyc = 0
    for cyc in range(1, args.converge_max + 1):
        s.cycle(cyc)
        r = s.residuals()[0][0]
        r0 = r0 or r
        if r <= 1e-8 * r0:
            break
    secs = time.perf_counter() - t0
    f = s.forces()
    s.close()
    d = mesh.level(1)
    name = f"{nx}x{ny}x{nz} hex -> 6 tets ({d.n_nodes:,} nodes, {d.n_sides:,} edges)"
    cpu = None if args.no_cpu_baseline else cpu_baseline(mesh, c, u0, cycles=args.cpu_cycles,
                                                          sample_of=f"the same {d.n_nodes:,}-node upwind workload")
    print(json.dumps({
        "metric": METRIC, "value": args.steps / (ms / 1e3), "unit": "cycles/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (generated bump channel, seeded +-1% density)",
        "config": {"workload": "inviscid Euler, M 0.5, CFL 2, on the bump channel " + name + ", 3 agglomerated "
                               "MG levels, growing V-cycle; the upwind extension (no reference counterpart): "
                               "Roe flux, MUSCL from Galerkin gradients with the Van Albada limiter on level 1, "
                               "5 stages (1/4, 1/6, 3/8, 1/2, 1)",
                   "mesh_nodes": d.n_nodes, "mesh_edges": d.n_sides, "levels": mesh.nlevels},
        "converge": {"seconds": secs, "cycles": cyc, "reached": bool(r <= 1e-8 * r0),
                     "log10_reduction": float(math.log10(r / r0)), "CL": float(f[0]), "CD": float(f[1])},
        "cpu_baseline": cpu, "gpu_launches": launches,
    }), flush=True)


def run_adjoint(args):
    """The adjoint configuration for the central flux: dCL/dX and
    dCD/dX along the normal displacement of wall nodes of the bump channel
    48x16x16 hex -> tets (the Euler configuration's mesh) with its interior
    nodes jittered by up to 15% of the spacing (seed 11: no two edges tie in
    the dissipation's min/max switches), inviscid (or laminar with
    --adjoint-re, adiabatic walls), M 0.5, central flux + JST, CFL 2, 3
    levels, FP64.  The primal is converged to a residual of 1e-15,
    the adjoint to 1e-12; then central differences of converged solutions on
    moved meshes at 32 seeded wall nodes (SplitMix64 seed 4), step 1e-7 of
    the channel height.  One JSON line: the adjoint solve's seconds, beside
    the primal solve's and the finite-difference agreement."""
    import torch
    import flite3d_b200 as F
    from flite3d_b200.mesh import splitmix64
    if not torch.cuda.is_available():
        raise SystemExit("no CUDA device: the product path has no CPU fallback")
    nx, ny, nz = [int(v) for v in args.adjoint_mesh.split(",")]
    nlev = 3 if nx * ny * nz <= 48 * 16 * 16 else 4
    base = F.Mesh.bump_channel(nx, ny, nz, 0.05, nlevels=nlev)
    X = base.array(1, "coords")
    jit = np.random.default_rng(11).uniform(-1, 1, X.shape) * 0.15 / nz
    jit[:, :base.level(1).n_bnodes] = 0.0
    X = X + jit
    at = lambda Y: base.with_level1_geometry(*base.geometry(Y))
    mesh = at(X)
    re = args.adjoint_re
    c = F.default_controls(ReynoldsNumber=re, fluxType=1, CFLNumber=2.0, multigridScheme=3,
                           numberOfGridsToUse=nlev, wallsAreIsentropic=1, viscosityScheme=1)
    flow = f"laminar Re {re:g}, adiabatic walls" if re > 0 else "inviscid"

    def converge(m, u0=None, tol=1e-15, max_cycles=args.adjoint_primal_cycles):
        s = F.Solver(c, m)
        s.set_state(F.initial_state(c, m) if u0 is None else u0)
        s.start()
        res, it = None, 0
        for it in range(1, max_cycles + 1):
            s.cycle(it)
            if it % 50 == 0:
                res = s.residuals()[0][0]
                if res < tol:
                    break
        return s, res, it

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s, res, ncyc = converge(mesh)
    torch.cuda.synchronize()
    t_primal = time.perf_counter() - t0
    u = s.get_state(1)
    out = {}
    for name in ("CL", "CD"):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = s.adjoint_solve(name, tol=1e-12, max_iter=args.adjoint_max_iter)
        torch.cuda.synchronize()
        out[name] = (r, time.perf_counter() - t0,
                     base.geometry_vjp(r["side_w_bar"], r["bnd_w_bar"], r["volume_bar"], xyz=X))
    # the same CL adjoint by the plain fixed-point iteration, for comparison
    # (on the Euler mesh; on larger ones it takes too long for a bench run)
    fixed = None
    if nx * ny * nz <= 48 * 16 * 16:
        s.set_adjoint_method("fixed-point")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rf = s.adjoint_solve("CL", tol=1e-12, max_iter=400000)
        torch.cuda.synchronize()
        t_fixed = time.perf_counter() - t0
        s.set_adjoint_method("gmres")
        xf = base.geometry_vjp(rf["side_w_bar"], rf["bnd_w_bar"], rf["volume_bar"], xyz=X)
        fixed = {"seconds": t_fixed, "iterations": rf["iterations"], "residual": rf["residual"],
                 "max_rel_diff_dCL_dX_vs_gmres": float(np.abs(xf - out["CL"][2]).max() /
                                                        np.abs(out["CL"][2]).max())}
    reg, ind = base.array(1, "node_reg"), base.array(1, "node_ind")
    wall = ind[reg[0] - 1:reg[1]] - 1
    bw, bidx = base.array(1, "bnd_w"), base.array(1, "bnd_idx")
    a = np.zeros_like(X)
    for k in range(2):
        np.add.at(a, (slice(None), bidx[k] - 1), -bw)
    nrm = a / np.linalg.norm(a, axis=0).clip(1e-300)
    pick = (splitmix64(4, 64) % np.uint64(len(wall))).astype(np.int64)
    nodes = list(dict.fromkeys(wall[pick].tolist()))[:args.adjoint_nodes]
    h = 1e-7
    errs = {"CL": [], "CD": []}
    t0 = time.perf_counter()
    for k in nodes:
        dX = np.zeros_like(X)
        dX[:, k] = nrm[:, k] * h
        sp = converge(at(X + dX), u0=u, max_cycles=3000)[0]
        sm = converge(at(X - dX), u0=u, max_cycles=3000)[0]
        for name in ("CL", "CD"):
            fd = (sp.objective(name) - sm.objective(name)) / (2 * h)
            adj = float((out[name][2][:, k] * nrm[:, k]).sum())
            errs[name].append(abs(adj - fd) / max(abs(fd), 1e-300))
    t_fd = time.perf_counter() - t0
    d = mesh.level(1)
    rl = out["CL"][0]
    print(json.dumps({
        "metric": "adjoint dCL/dX solve time", "value": out["CL"][1], "unit": "s", "n_gpus": 1,
        "steps": 1, "warmup": 0, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (generated bump-channel mesh, jittered interior nodes, freestream start)",
        "config": {"workload": f"steady adjoint of CL and CD, {flow}, M 0.5, central flux + JST, on the bump "
                               f"channel {nx}x{ny}x{nz} hex -> 6 tets with interior nodes jittered by 15% of the "
                               f"spacing, {nlev} agglomerated MG levels for the primal, FP64",
                   "mesh_nodes": d.n_nodes, "mesh_edges": d.n_sides},
        "primal": {"seconds": t_primal, "cycles": ncyc, "residual": res},
        "adjoint": {name: {"J": out[name][0]["J"], "seconds": out[name][1], "iterations": out[name][0]["iterations"],
                           "residual": out[name][0]["residual"]} for name in out},
        "adjoint_over_primal_time": out["CL"][1] / t_primal,
        "ms_per_transpose_product": 1e3 * out["CL"][1] / max(out["CL"][0]["iterations"], 1),
        "ms_per_primal_cycle": 1e3 * t_primal / ncyc,
        "method": "GMRES(50) on (I - P G_u^T) lam = P J_u^T",
        "fixed_point": fixed,
        "fd_check": {"nodes": len(nodes), "step": h, "seconds": t_fd,
                     "max_rel_err": {n: max(e) for n, e in errs.items()},
                     "median_rel_err": {n: float(np.median(e)) for n, e in errs.items()}} if nodes else None,
        "gpu_launches": None,
    }), flush=True)


def small_batch(args, ncases=64, size=(48, 16, 16)):
    """Many small solves, where launches dominate: the c1 mesh (bump
    48x16x16, 3 levels) x 64 conditions, inviscid FP64, with case groups and
    with a graph per case."""
    import flite3d_b200 as F
    from flite3d_b200.mesh import splitmix64
    from flite3d_b200.solver import Batch
    m = F.Mesh.bump_channel(*size, 0.05, 3)
    bits = splitmix64(9, 2 * ncases) >> np.uint64(11)
    uni = bits.astype(np.float64) / float(1 << 53)
    cases = [(F.default_controls(ReynoldsNumber=0.0, MachNumber=0.3 + 0.5 * uni[2 * k + 1],
                                 alpha=-4.0 + 12.0 * uni[2 * k], CFLNumber=2.0, fluxType=1, multigridScheme=3,
                                 numberOfGridsToUse=3), m) for k in range(ncases)]
    out = {"workload": f"bump {size} x {ncases} conditions, inviscid, FP64, 3 levels", "nodes": m.level(1).n_nodes}
    for on in (True, False):
        batch = Batch(cases)
        batch.set_grouping(on)
        for (c, mm), s in zip(cases, batch.cases):
            s.set_state(F.initial_state(c, mm))
            s.start()
        batch.time_cycles(args.warmup)
        ms, launches = batch.time_cycles(args.steps, cycle_no=args.warmup + 1, sequential=False)
        out["case_groups" if on else "graph_per_case"] = {
            "value": ncases * args.steps / (ms / 1e3), "unit": "case-cycles/s", "ms_per_step": ms / args.steps,
            "kernel_launches_per_batch_cycle": launches}
        batch.close()
    m.close()
    out["groups_vs_graph_per_case"] = out["case_groups"]["value"] / out["graph_per_case"]["value"]
    return out


def run_batch(args):
    """Batched solves: the bump channel at 120x40x40, 192x64x64 and
    264x88x88 hexes x 16 flow conditions each (angle of attack uniform in
    [-4, 8] degrees, Mach uniform in [0.3, 0.8], SplitMix64 seed 5), inviscid,
    FLITE_MIXED.  One JSON line: case-cycles per second of one graph launch
    per batch cycle (the cases on one mesh as a case group: every kernel of
    the cycle launched once for all of them), against the same graph with a
    branch per case and against the cases' graphs launched one after
    another."""
    import torch
    import flite3d_b200 as F
    from flite3d_b200.mesh import splitmix64
    from flite3d_b200.solver import Batch
    if not torch.cuda.is_available():
        raise SystemExit("no CUDA device: the product path has no CPU fallback")
    sizes = [(120, 40, 40), (192, 64, 64), (264, 88, 88)][:args.batch_meshes]
    meshes = [F.Mesh.bump_channel(nx, ny, nz, 0.05, 4) for nx, ny, nz in sizes]
    bits = splitmix64(5, 2 * args.batch_conditions) >> np.uint64(11)
    uni = bits.astype(np.float64) / float(1 << 53)
    cases = []
    for m in meshes:
        for k in range(args.batch_conditions):
            alpha = -4.0 + 12.0 * uni[2 * k]
            mach = 0.3 + 0.5 * uni[2 * k + 1]
            c = F.default_controls(ReynoldsNumber=0.0, MachNumber=mach, alpha=alpha, CFLNumber=2.0,
                                   fluxType=1, multigridScheme=3, numberOfGridsToUse=4, precision=1)
            cases.append((c, m))
    batch = Batch(cases)
    for (c, m), s in zip(cases, batch.cases):
        s.set_state(F.initial_state(c, m))
        s.start()
    e, nb, best, lanes, best_lanes = 256, 256, None, None, None
    if not args.batch_no_autotune:
        e, nb, best = batch.autotune(reps=2)
        lanes, best_lanes = batch.autotune_lanes(reps=2)
    if args.batch_grouping != "auto":  # the mode asked for in place of the tuner's
        batch.set_grouping(args.batch_grouping == "on")
    grouped = batch.grouping()
    for (c, m), s in zip(cases, batch.cases):
        s.set_state(F.initial_state(c, m))
        s.start()
    batch.time_cycles(args.warmup)
    ms_g, launches = batch.time_cycles(args.steps, cycle_no=args.warmup + 1, sequential=False)
    groups = batch.groups()
    # the other grouping mode, and the cases' graphs one after another
    batch.set_grouping(not grouped)
    ms_o, launches_o = batch.time_cycles(args.steps, cycle_no=args.warmup + args.steps + 1, sequential=False)
    ms_s, _ = batch.time_cycles(args.steps, cycle_no=args.warmup + 2 * args.steps + 1, sequential=True)
    batch.close()
    small = None if args.no_small_batch else small_batch(args)
    n = len(cases)
    print(json.dumps({
        "metric": "batched MG case-cycles/s", "value": n * args.steps / (ms_g / 1e3), "unit": "case-cycles/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_g / args.steps,
        "higher_is_better": True, "dtype": "f32 flux increments / f64", "data": "synthetic",
        "config": {"workload": f"{len(meshes)} bump-channel meshes {sizes} x {args.batch_conditions} "
                               "conditions (alpha U[-4,8] deg, M U[0.3,0.8]), inviscid, FLITE_MIXED",
                   "cases": n, "mesh_nodes": [m.level(1).n_nodes for m in meshes]},
        "case_groups": groups,
        "grouping": {"chosen": "case groups" if grouped else "a graph per case",
                     "other": {"value": n * args.steps / (ms_o / 1e3), "ms_per_step": ms_o / args.steps,
                               "kernel_launches_per_batch_cycle": launches_o}},
        "sequential": {"value": n * args.steps / (ms_s / 1e3), "ms_per_step": ms_s / args.steps},
        "graph_vs_sequential": ms_s / ms_g, "kernel_launches_per_batch_cycle": launches,
        "small_meshes": small,
        "autotune": {"edge_block": e, "node_block": nb, "best_ms": best, "lanes_per_level": lanes,
                     "best_ms_lanes": best_lanes},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-cycles", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mesh", default=None, help="NX,NY,NZ hexes (default 264,88,88)")
    ap.add_argument("--no-mixed", action="store_true", help="skip the FLITE_MIXED cycle rate")
    ap.add_argument("--kernel-options", default=None,
                    help="NODE_BLOCK,UNROLL,LANES_L1,...: fixed launch options instead of tuning them")
    ap.add_argument("--node-order", type=int, default=0,
                    help="device node numbering: 0 the mesh's own, 1 the locality (Morton) order")
    ap.add_argument("--tiled-modes", default=None,
                    help="with --kernel-options: TILED_L1,TILED_L2,... (0 off, 1 or 2 on; default 1)")
    ap.add_argument("--fusion", default=None,
                    help="with --kernel-options: per level 1 to share the walks of gathers over the same "
                         "incidence list, 0 for separate kernels (default 1)")
    ap.add_argument("--no-converge", action="store_true",
                    help="skip the time to a 1e-8 residual reduction, FP64 and FLITE_MIXED")
    ap.add_argument("--parity-cycles", type=int, default=2,
                    help="cycles of the GPU-vs-CPU-restatement check on the bench mesh (0: none)")
    ap.add_argument("--converge-max", type=int, default=3000)
    ap.add_argument("--batch", action="store_true", help="the batched multi-condition workload instead")
    ap.add_argument("--rans", action="store_true", help="the RANS (Spalart-Allmaras, NACA0012) workload instead")
    ap.add_argument("--rans-ni", type=int, default=200)
    ap.add_argument("--rans-nj", type=int, default=120)
    ap.add_argument("--rans-nk", type=int, default=240)
    ap.add_argument("--adjoint", action="store_true",
                    help="the steady adjoint (dCL/dX, dCD/dX) workload with its finite-difference check")
    ap.add_argument("--adjoint-nodes", type=int, default=32, help="wall nodes of the finite-difference check")
    ap.add_argument("--adjoint-mesh", default="48,16,16", help="NX,NY,NZ hexes of the adjoint workload")
    ap.add_argument("--adjoint-re", type=float, default=0.0, help="Reynolds number (0: inviscid)")
    ap.add_argument("--adjoint-primal-cycles", type=int, default=6000)
    ap.add_argument("--adjoint-max-iter", type=int, default=400000,
                    help="products with the transposed iteration Jacobian per adjoint solve")
    ap.add_argument("--upwind", action="store_true",
                    help="the bump-channel Euler case with the upwind Roe / MUSCL / Van Albada, five-stage "
                         "extension instead")
    ap.add_argument("--upwind-mesh", default="48,16,16", help="NX,NY,NZ hexes of the upwind workload")
    ap.add_argument("--batch-meshes", type=int, default=3)
    ap.add_argument("--batch-conditions", type=int, default=16)
    ap.add_argument("--batch-grouping", default="auto", choices=["auto", "on", "off"],
                    help="case groups on or off, or the autotuner's choice")
    ap.add_argument("--no-small-batch", action="store_true", help="skip the batch of small meshes")
    ap.add_argument("--batch-no-autotune", action="store_true", help="default block sizes and gather tiles")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.mesh:
        MESH["nx"], MESH["ny"], MESH["nz"] = [int(v) for v in args.mesh.split(",")]
    if args.impl == "reference":
        run_reference(args)
    elif args.batch:
        run_batch(args)
    elif args.rans:
        run_rans(args)
    elif args.adjoint:
        run_adjoint(args)
    elif args.upwind:
        run_upwind(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
