"""ctypes mirror of the C ABI in include/flite_gpu.h and include/flite_prepro.h.

The structures here must match the C declarations field for field; the
loaders locate the in-tree shared libraries built by flite3d_b200.build.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))

FLITE_OK = 0
FLITE_EINVAL = 1
FLITE_EUNSUPPORTED = 2
FLITE_ENAN = 3
FLITE_ETIMEOUT = 4
FLITE_ECUDA = 5
FLITE_ENOMEM = 6
FLITE_EIO = 7
FLITE_FP64 = 0
FLITE_MIXED = 1
FLITE_RECON_NONE = 0
FLITE_RECON_VAN_ALBADA = 1

_d, _i = ctypes.c_double, ctypes.c_int

_CONTROL_FIELDS = [
    # freestream and physics
    ("MachNumber", _d), ("alpha", _d), ("beta", _d), ("ReynoldsNumber", _d),
    ("PrandtlNumber", _d), ("gamma", _d), ("inflowTemperature", _d), ("wallTemperature", _d),
    ("wallsAreIsentropic", _i), ("fluxType", _i), ("HLLCFluxOrder", _i), ("HLLCClipping", _d),
    ("Automaticlipping", _i), ("GradientMethod", _i), ("dissipationScheme", _i),
    ("coarseGridDissipationScheme", _i), ("secondOrderDissipationFactor", _d),
    ("fourthOrderDissipationFactor", _d), ("coarseGridDissipationFactor", _d),
    ("useMatrixDissipation", _i), ("HartensCorrectionFactor", _d),
    ("useDissipationWeighting", _i), ("viscosityScheme", _i), ("boundaryTerm", _i),
    # time stepping and multigrid
    ("CFLNumber", _d), ("turbulentCFLNumber", _d), ("turbK", _d), ("maxIncrementFactor", _d),
    ("minimumDensity", _d), ("multigridScheme", _i), ("numberOfRelaxationSteps", _i),
    ("numberOfGridsToUse", _i), ("multigridBCRelaxation", _d), ("prolongationRelaxation", _d),
    ("turbProlongationRelaxation", _d), ("prolongationMappingScheme", _i),
    ("numberOfMGIterations", _i), ("maximumnumberofcycles", _i), ("writeToFileInterval", _i),
    ("initialResidual", _d), ("numberOfCFLIncrements", _i),
    # turbulence and bookkeeping
    ("turbulenceModel", _i), ("numberOfTurbulenceGrids", _i), ("numberOfTurbulenceSteps", _i),
    ("tripFactor", _d), ("triggerRadius", _d), ("turbulenceTriggerValue", _d),
    ("numberOfTriggerSteps", _i), ("maxTurbulenceValue", _d), ("turbulentPrandtlNumber", _d),
    ("referenceArea", _d), ("datum", _d * 3), ("groundplane", _d), ("forceCalcType", _i),
    ("restartNumber", _i), ("numberOfProcesses", _i),
    # rejected unless at their steady default
    ("flowType", _i), ("explicit_", _i), ("SAS", _i), ("GUSTMODEL", _i), ("movingwall", _i),
    ("patchInitialization", _i), ("nspan", _i), ("timeScheme", _i), ("numberOfRSSteps", _i),
    ("numberOfPSSteps", _i), ("residualSmoothingFactor", _d),
    ("prolongationSmoothingFactor", _d), ("physicalTimeStep", _d), ("engineBCRelaxation", _d),
    ("engineFlowType", _i), ("numberOfEORelaxationSteps", _i), ("enginesFrontMassFlow", _d * 2),
    ("enginesRearParameters", _d * 14),
    ("inflowField", _d * 12),
    ("precision", _i), ("reconstruction", _i), ("rungeKuttaStages", _i),
]


class Controls(ctypes.Structure):
    _fields_ = _CONTROL_FIELDS

    def as_dict(self):
        out = {}
        for name, typ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(v, "__len__") else v
        return out


_P = ctypes.c_void_p


class LevelDesc(ctypes.Structure):
    _fields_ = [
        ("n_nodes", ctypes.c_int32), ("n_sides", ctypes.c_int32), ("n_bsides", ctypes.c_int32),
        ("n_bnodes", ctypes.c_int32), ("n_normals", ctypes.c_int32),
        ("side_idx", _P), ("side_w", _P), ("side_len", _P), ("bnd_idx", _P), ("bnd_w", _P),
        ("node_reg", _P), ("node_ind", _P), ("volume", _P), ("wall_dist", _P), ("coords", _P),
        ("coord_move", _P), ("parent", _P), ("rweight", _P),
        ("side_gcl", _P), ("bnd_gcl", _P), ("volume_prev", _P), ("volume_prev2", _P),
        ("n_engine_sides", ctypes.c_int32), ("engine_idx", _P), ("engine_w", _P),
    ]


GPU_SYMBOLS = [
    "flite_controls_default", "flite_controls_derive", "flite_create", "flite_destroy",
    "flite_last_error", "flite_set_state", "flite_get_state", "flite_get_pressure",
    "flite_init_freestream", "flite_start", "flite_do_time_iterations", "flite_restrict",
    "flite_prolong", "flite_map_fine_to_coarse", "flite_cycle", "flite_residuals",
    "flite_forces", "flite_residual_fwd", "flite_time_cycles", "flite_cycle_launches",
    "flite_profile_level", "flite_batch_create", "flite_batch_destroy", "flite_batch_context",
    "flite_batch_cycle", "flite_batch_run", "flite_batch_time_cycles", "flite_batch_autotune", "flite_batch_set_blocks", "flite_batch_set_grouping", "flite_batch_groups", "flite_batch_grouping",
    "flite_batch_autotune_lanes", "flite_explicit_time_step",
    "flite_residual_vjp", "flite_profile_adjoint", "flite_profile_kernels", "flite_set_kernel_options", "flite_set_gather_lanes",
    "flite_iteration_vjp", "flite_adjoint_solve", "flite_objective", "flite_set_adjoint_method",
    "flite_next_physical_step", "flite_set_node_order", "flite_set_tiled_gather", "flite_set_gather_fusion", "flite_update_geometry",
]

PREPRO_SYMBOLS = [
    "fp_bump_channel", "fp_naca0012", "fp_from_tets", "fp_free", "fp_num_levels", "fp_level_desc",
    "fp_node_perm", "fp_check", "fp_geometry", "fp_geometry_vjp", "fp_write_sol", "fp_read_sol", "fp_write_rst", "fp_read_rst",
    "fp_write_res", "fp_write_unk", "fp_read_unk", "fp_write_plotreg", "fp_makeplot", "fp_write_plt",
    "fp_read_inp", "fp_parse_inp_text", "fp_rsd_line", "fp_append_rsd", "fp_cycle_line",
    "fp_controls_default", "fp_controls_derive", "fp_set_moving_geometry", "fp_coordinate_movement", "fp_gcl_check",
    "fp_canonical", "fp_partition", "fp_write_sol_domains", "fp_read_sol_domains", "fp_from_elements",
]

_libs = {}


def lib_path(name):
    return os.path.join(_HERE, name)


def load(name):
    """Load an in-tree shared library once (RTLD_GLOBAL off, by path)."""
    if name not in _libs:
        path = lib_path(name)
        if not os.path.exists(path):
            raise OSError(
                f"{path} is missing: build the native libraries with "
                "`python -c 'import flite3d_b200.build as b; b.build_all()'`")
        _libs[name] = ctypes.CDLL(path)
    return _libs[name]


def gpu_lib():
    return load("libflite_gpu.so")


def prepro_lib():
    return load("libflite_prepro.so")


def check(rc, what="call", ctx_err=None):
    if rc != FLITE_OK:
        msg = f"{what} failed with status {rc}"
        if ctx_err:
            msg += f": {ctx_err}"
        raise RuntimeError(msg)
