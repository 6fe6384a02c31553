"""ctypes binding of the C ABI declared in include/fvh.h (libfvh.so).

The library is loaded from fvhoe_b200/_lib/libfvh.so. There is no fallback:
if the library is missing the import of this module raises, naming the
build command.
"""

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libfvh.so")

ABI_VERSION = 3

OK = 0
ERR_CONFIG = -1
ERR_CUDA = -2
ERR_TIMEOUT = -3
ERR_NONFINITE = -4
ERR_ARG = -5

DMR_Y0 = "special-case-double-mach-reflection-y=0"
BC = {"periodic": 0, "outflow": 1, "reflective": 2, "free": 3, "dirichlet": 4, DMR_Y0: 5}
RIEMANN = {"hllc": 0, "llf": 1, "advection_upwind": 2}
LIMITER = {"minmod": 0, "moncen": 1, None: 2}
PRECISION = {"fp64": 0, "fp32": 1}
INTEGRATOR = {"euler": 0, "ssprk2": 1, "ssprk3": 2, "rk4": 3}

# every symbol include/fvh.h declares
EXPORTS = (
    "fvh_config_default",
    "fvh_create",
    "fvh_destroy",
    "fvh_last_error",
    "fvh_scratch_bytes",
    "fvh_rhs",
    "fvh_step",
    "fvh_stage",
    "fvh_step_host",
    "fvh_host_sync",
    "fvh_primitives",
    "fvh_trouble_flags",
    "fvh_trouble_log",
    "fvh_set_log_mode",
    "fvh_set_log_divisor",
    "fvh_get_stats",
    "fvh_kernel_launches",
    "fvh_profile_enable",
    "fvh_profile_read",
    "fvh_primitives_noalloc",
    "fvh_primitives_noalloc_max_doubles",
    "fvh_primitives_noalloc_error",
    "fvh_mlp_param_count",
    "fvh_mlp_create",
    "fvh_mlp_destroy",
    "fvh_mlp_last_error",
    "fvh_mlp_get_params",
    "fvh_mlp_set_params",
    "fvh_mlp_features",
    "fvh_mlp_train_step",
    "fvh_mlp_gradients",
    "fvh_mlp_logits",
    "fvh_mlp_errors",
    "fvh_set_predictor",
    "fvh_set_predictor_interval",
    "fvh_get_pred_stats",
    "fvh_pred_flags",
    "fvh_boundary_layout",
    "fvh_set_boundary_values",
    "fvh_ensemble_create",
    "fvh_ensemble_destroy",
    "fvh_ensemble_last_error",
    "fvh_ensemble_bytes",
    "fvh_ensemble_state",
    "fvh_ensemble_load",
    "fvh_ensemble_store",
    "fvh_ensemble_reset",
    "fvh_ensemble_step",
    "fvh_ensemble_status",
    "fvh_ensemble_configure",
    "fvh_ensemble_variant_info",
    "fvh_ensemble_autotune",
    "fvh_ensemble_graph_info",
    "fvh_ensemble_set_wait_limit",
)

KERNEL_KINDS = ("centre", "transverse", "face", "candidate", "detect", "fallback", "final", "small", "predict")

MLP_FEATURES = 100
MLP_ROW = 112


class FvhConfig(ctypes.Structure):
    """Mirror of struct fvh_config (include/fvh.h)."""

    _fields_ = [
        ("abi_version", ctypes.c_int),
        ("nvars", ctypes.c_int),
        ("n", ctypes.c_int * 3),
        ("p", ctypes.c_int * 3),
        ("h", ctypes.c_double * 3),
        ("gamma", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("csq_floor", ctypes.c_double),
        ("use_fixed_dt", ctypes.c_int),
        ("fixed_dt", ctypes.c_double),
        ("riemann", ctypes.c_int),
        ("bc", (ctypes.c_int * 2) * 3),
        ("a_posteriori", ctypes.c_int),
        ("slope_limiter", ctypes.c_int),
        ("force_trouble", ctypes.c_int),
        ("nad_eps", ctypes.c_double),
        ("nad_global", ctypes.c_int),
        ("nad_relative", ctypes.c_int),
        ("nad_var_mask", ctypes.c_int),
        ("pad_var", ctypes.c_int),
        ("pad_lo", ctypes.c_double),
        ("pad_hi", ctypes.c_double),
        ("sed", ctypes.c_int),
        ("sed_eps", ctypes.c_double),
        ("convex", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("log_troubles", ctypes.c_int),
        ("device", ctypes.c_int),
        ("kernel_path", ctypes.c_int),
        ("dmr_split", ctypes.c_int),
    ]


PATH = {"auto": 0, "generic": 1, "fused2d": 2}


class FvhStats(ctypes.Structure):
    """Mirror of struct fvh_stats (include/fvh.h)."""

    _fields_ = [
        ("dt_stage", ctypes.c_double),
        ("dt_step", ctypes.c_double),
        ("troubled", ctypes.c_uint),
        ("nonfinite", ctypes.c_uint),
    ]


class FvhPredStats(ctypes.Structure):
    """Mirror of struct fvh_pred_stats (include/fvh.h)."""

    _fields_ = [
        ("predicted", ctypes.c_uint),
        ("troubled", ctypes.c_uint),
        ("missed", ctypes.c_uint),
        ("false_alarm", ctypes.c_uint),
        ("revised_faces", ctypes.c_uint),
        ("flux_fallback_faces", ctypes.c_uint),
    ]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing; build it with `python -m fvhoe_b200.build` "
            "(there is no CPU fallback for the CUDA backend)"
        )
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    dp = ctypes.POINTER(ctypes.c_double)
    lib.fvh_config_default.argtypes = [ctypes.POINTER(FvhConfig)]
    lib.fvh_config_default.restype = None
    lib.fvh_create.argtypes = [ctypes.POINTER(FvhConfig), ctypes.POINTER(vp)]
    lib.fvh_destroy.argtypes = [vp]
    lib.fvh_last_error.argtypes = [vp]
    lib.fvh_last_error.restype = ctypes.c_char_p
    lib.fvh_scratch_bytes.argtypes = [vp]
    lib.fvh_scratch_bytes.restype = ctypes.c_size_t
    lib.fvh_rhs.argtypes = [vp, vp, vp, dp, vp]
    lib.fvh_step.argtypes = [vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, dp, vp]
    lib.fvh_stage.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                              dp, vp]
    lib.fvh_step_host.argtypes = [vp, vp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, dp, vp]
    lib.fvh_host_sync.argtypes = [vp]
    lib.fvh_primitives.argtypes = [vp, vp, vp, ctypes.c_int, vp]
    lib.fvh_trouble_flags.argtypes = [vp, vp, vp]
    lib.fvh_trouble_log.argtypes = [vp, ctypes.c_double, vp, vp, vp, vp]
    lib.fvh_set_log_mode.argtypes = [vp, ctypes.c_int]
    lib.fvh_set_log_divisor.argtypes = [vp, ctypes.c_double]
    lib.fvh_set_log_divisor.restype = ctypes.c_int
    lib.fvh_get_stats.argtypes = [vp, ctypes.POINTER(FvhStats), vp]
    lib.fvh_kernel_launches.argtypes = []
    lib.fvh_kernel_launches.restype = ctypes.c_uint64
    lib.fvh_profile_enable.argtypes = [vp, ctypes.c_int]
    lib.fvh_profile_read.argtypes = [vp, dp, dp, ctypes.POINTER(ctypes.c_uint64), vp]
    lib.fvh_primitives_noalloc.argtypes = [ctypes.POINTER(FvhConfig), vp, vp, ctypes.c_int, vp]
    lib.fvh_primitives_noalloc.restype = ctypes.c_int
    lib.fvh_primitives_noalloc_max_doubles.argtypes = []
    lib.fvh_primitives_noalloc_max_doubles.restype = ctypes.c_size_t
    lib.fvh_primitives_noalloc_error.argtypes = []
    lib.fvh_primitives_noalloc_error.restype = ctypes.c_char_p
    fp = ctypes.POINTER(ctypes.c_float)
    lib.fvh_mlp_param_count.argtypes = []
    lib.fvh_mlp_param_count.restype = ctypes.c_size_t
    lib.fvh_mlp_create.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(vp)]
    lib.fvh_mlp_destroy.argtypes = [vp]
    lib.fvh_mlp_last_error.argtypes = [vp]
    lib.fvh_mlp_last_error.restype = ctypes.c_char_p
    lib.fvh_mlp_get_params.argtypes = [vp, fp, ctypes.c_size_t]
    lib.fvh_mlp_set_params.argtypes = [vp, fp, ctypes.c_size_t]
    lib.fvh_mlp_features.argtypes = [vp, vp, vp, vp]
    lib.fvh_mlp_train_step.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_float, ctypes.c_float, fp, vp]
    lib.fvh_mlp_gradients.argtypes = [vp, vp, vp, ctypes.c_int, ctypes.c_float, vp, fp, vp]
    lib.fvh_mlp_logits.argtypes = [vp, vp, ctypes.c_int, vp, vp]
    lib.fvh_mlp_errors.argtypes = [vp]
    lib.fvh_mlp_errors.restype = ctypes.c_uint
    lib.fvh_set_predictor.argtypes = [vp, vp, ctypes.c_float]
    lib.fvh_set_predictor_interval.argtypes = [vp, ctypes.c_int]
    lib.fvh_get_pred_stats.argtypes = [vp, ctypes.POINTER(FvhPredStats), vp]
    lib.fvh_pred_flags.argtypes = [vp, vp, vp]
    ip = ctypes.POINTER(ctypes.c_int)
    up = ctypes.POINTER(ctypes.c_uint)
    lib.fvh_boundary_layout.argtypes = [vp, ctypes.c_int, ctypes.c_int, ip, ip, ctypes.POINTER(ctypes.c_size_t)]
    lib.fvh_boundary_layout.restype = ctypes.c_int
    lib.fvh_set_boundary_values.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp]
    lib.fvh_set_boundary_values.restype = ctypes.c_int
    lib.fvh_ensemble_create.argtypes = [ctypes.POINTER(FvhConfig), ctypes.c_int, ip, ip, dp, dp, ctypes.POINTER(vp)]
    lib.fvh_ensemble_destroy.argtypes = [vp]
    lib.fvh_ensemble_last_error.argtypes = [vp]
    lib.fvh_ensemble_last_error.restype = ctypes.c_char_p
    lib.fvh_ensemble_bytes.argtypes = [vp]
    lib.fvh_ensemble_bytes.restype = ctypes.c_size_t
    lib.fvh_ensemble_state.argtypes = [vp, ctypes.c_int]
    lib.fvh_ensemble_state.restype = vp
    lib.fvh_ensemble_load.argtypes = [vp, ctypes.c_int, vp, vp]
    lib.fvh_ensemble_store.argtypes = [vp, ctypes.c_int, vp, vp]
    lib.fvh_ensemble_reset.argtypes = [vp, ctypes.c_double, ctypes.c_double, vp]
    lib.fvh_ensemble_step.argtypes = [vp, ctypes.c_int, vp]
    lib.fvh_ensemble_status.argtypes = [vp, dp, ip, ip, up, vp]
    lib.fvh_ensemble_configure.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.fvh_ensemble_variant_info.argtypes = [vp, ctypes.c_int, ip, ip, ip, ctypes.POINTER(ctypes.c_size_t)]
    lib.fvh_ensemble_autotune.argtypes = [vp, ctypes.c_int, ip, ip, dp, vp]
    lib.fvh_ensemble_graph_info.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_char_p)]
    lib.fvh_ensemble_set_wait_limit.argtypes = [vp, ctypes.c_uint]
    for name in ("fvh_ensemble_create", "fvh_ensemble_destroy", "fvh_ensemble_load", "fvh_ensemble_store",
                 "fvh_ensemble_reset", "fvh_ensemble_step",
                 "fvh_ensemble_status", "fvh_ensemble_configure", "fvh_ensemble_variant_info",
                 "fvh_ensemble_autotune", "fvh_ensemble_graph_info", "fvh_ensemble_set_wait_limit"):
        getattr(lib, name).restype = ctypes.c_int
    for name in ("fvh_create", "fvh_destroy", "fvh_rhs", "fvh_step", "fvh_stage", "fvh_step_host", "fvh_host_sync",
                 "fvh_primitives", "fvh_trouble_flags",
                 "fvh_trouble_log", "fvh_set_log_mode", "fvh_get_stats", "fvh_profile_enable", "fvh_profile_read",
                 "fvh_mlp_create", "fvh_mlp_destroy", "fvh_mlp_get_params", "fvh_mlp_set_params", "fvh_mlp_features",
                 "fvh_mlp_train_step", "fvh_mlp_gradients", "fvh_mlp_logits", "fvh_set_predictor",
                 "fvh_set_predictor_interval", "fvh_get_pred_stats", "fvh_pred_flags"):
        getattr(lib, name).restype = ctypes.c_int
    return lib


lib = _load()


class FvhError(RuntimeError):
    """A non-zero status from the library, with its message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"fvh status {status}: {message}")
        self.status = status


class FvhNonFiniteError(FvhError, FloatingPointError):
    """FVH_ERR_NONFINITE: the update wrote NaN/Inf values, or its time step is
    not finite or not positive."""


def check(status: int, handle=None) -> None:
    if status != OK:
        msg = lib.fvh_last_error(handle)
        cls = FvhNonFiniteError if status == ERR_NONFINITE else FvhError
        raise cls(status, msg.decode() if msg else "")


def default_config() -> FvhConfig:
    cfg = FvhConfig()
    lib.fvh_config_default(ctypes.byref(cfg))
    return cfg
