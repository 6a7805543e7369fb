"""ctypes binding of libbia_b200.so (declarations in include/bia_capi.h).

The library is the product: every pair solve runs in its CUDA kernels.  Loading
fails loudly when the library has not been built; there is no CPU fallback.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbia_b200.so")

BIA_OK = 0
BIA_ERR_INVALID_ARGUMENT = 1
BIA_ERR_NONFINITE = 2
BIA_ERR_NOT_CONVERGED = 3
BIA_ERR_DEVICE_TIMEOUT = 4
BIA_ERR_CUDA = 5
BIA_ERR_OUT_OF_MEMORY = 6
BIA_ERR_NO_DEVICE = 7

METHOD_RKF = 0
METHOD_ALG = 1
METHOD_UNIVERSAL = 2
METHOD_LEARNED = 3


class BiaConfig(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int), ("itr", ctypes.c_int), ("eps_th", ctypes.c_double),
                ("dt", ctypes.c_double), ("err", ctypes.c_double),
                ("rkf_relerr", ctypes.c_double), ("rkf_abserr", ctypes.c_double),
                ("deterministic", ctypes.c_int)]


STAT_FIELDS = ("hyperbola", "parabola", "ellipse", "degenerate", "rkf", "universal",
               "iterations", "iter_hyperbola", "iter_ellipse", "iter_parabola", "iter_universal",
               "rkf_steps", "nonconverged", "bracket_exits", "fallbacks", "nonfinite",
               "learned", "learned_fallbacks", "learned_coarse", "timeouts", "learned_fp32_steps")


class BiaStats(ctypes.Structure):
    _fields_ = [(name, ctypes.c_longlong) for name in STAT_FIELDS]

    def as_dict(self):
        return {name: int(getattr(self, name)) for name in STAT_FIELDS}


class BiaDimStats(ctypes.Structure):
    _fields_ = [("accepted", ctypes.c_longlong), ("rejected", ctypes.c_longlong),
                ("nde", ctypes.c_int), ("ier", ctypes.c_int), ("h_last", ctypes.c_double),
                ("x_reached", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class BiaError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = status_string(status)
        super().__init__(f"{what}: {msg} (status {status})" if what else msg)


_lib = None
_D = ctypes.c_double
_I = ctypes.c_int
_V = ctypes.c_void_p
_PD = ctypes.POINTER(ctypes.c_double)


def lib():
    """Load libbia_b200.so; raises if it is missing (build it first)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m bia_3d_gpu_b200.build` "
                           "(the CUDA library is required; there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    L.bia_config_default.argtypes = [ctypes.POINTER(BiaConfig)]
    L.bia_config_default.restype = None
    L.bia_status_string.argtypes = [_I]
    L.bia_status_string.restype = ctypes.c_char_p
    L.bia_last_error.restype = _I
    L.bia_context_create.argtypes = [ctypes.POINTER(_V), _I, _V]
    L.bia_context_destroy.argtypes = [_V]
    L.bia_context_set_stream.argtypes = [_V, _V]
    L.bia_context_set_timing.argtypes = [_V, _I]
    L.bia_context_kernel_ms.argtypes = [_V, _PD, ctypes.POINTER(ctypes.c_longlong)]
    L.bia_step.argtypes = [_V, ctypes.POINTER(BiaConfig), _I] + [_V] * 8 + [ctypes.POINTER(BiaStats)]
    L.bia_run.argtypes = ([_V, ctypes.POINTER(BiaConfig), _I] + [_V] * 7 +
                          [_I, _I, ctypes.POINTER(BiaStats)])
    L.bia_run_host.argtypes = ([_V, ctypes.POINTER(BiaConfig), _I] + [_V] * 7 +
                               [_I, ctypes.POINTER(BiaStats)])
    L.bia_invariance.argtypes = [_V, _I, _D] + [_V] * 7 + [_PD]
    L.bia_measure_fp64_peak.argtypes = [_I, _PD]
    L.bia_context_stats.argtypes = [_V, ctypes.POINTER(BiaStats), _I]
    L.bia_shard_columns.argtypes = [_I, _I, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)]
    L.bia_shard_columns.restype = _I
    L.bia_step_shard.argtypes = ([_V, ctypes.POINTER(BiaConfig), _I] + [_V] * 7 + [_I, _I, _V,
                                 ctypes.POINTER(BiaStats)])
    L.bia_step_shard.restype = _I
    L.bia_apply_update.argtypes = [_V, _I, _D] + [_V] * 7
    L.bia_apply_update.restype = _I
    L.bia_step_noalloc.argtypes = [ctypes.POINTER(BiaConfig), _I] + [_V] * 9
    L.bia_step_noalloc.restype = _I
    L.bia_ensemble_create.argtypes = [_V, _I, ctypes.POINTER(ctypes.c_int), _PD, ctypes.POINTER(_V)]
    L.bia_ensemble_destroy.argtypes = [_V]
    L.bia_ensemble_particles.argtypes = [_V]
    L.bia_ensemble_particles.restype = ctypes.c_longlong
    L.bia_ensemble_run.argtypes = ([_V, _V, ctypes.POINTER(BiaConfig)] + [_V] * 7 +
                                   [_I, _I, ctypes.POINTER(BiaStats)])
    L.bia_ensemble_energy.argtypes = [_V, _V] + [_V] * 7 + [_PD]
    L.bia_ensemble_autotune.argtypes = ([_V, _V, ctypes.POINTER(BiaConfig)] + [_V] * 7 +
                                        [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)])
    L.bia_ensemble_autotune.restype = _I
    for name in ("bia_ensemble_create", "bia_ensemble_destroy", "bia_ensemble_run",
                 "bia_ensemble_energy"):
        getattr(L, name).restype = _I
    L.bia_context_autotune.argtypes = ([_V, ctypes.POINTER(BiaConfig), _I] + [_V] * 7 +
                                       [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_float)])
    L.bia_context_autotune.restype = _I
    L.bia_context_set_shape.argtypes = [_V, _I, _I, _I, _I]
    L.bia_context_set_shape.restype = _I
    L.bia_selftest_wait_timeout.argtypes = [_V]
    L.bia_selftest_wait_timeout.restype = _I
    L.bia_context_set_heads.argtypes = [_V, ctypes.c_char_p, ctypes.c_size_t]
    L.bia_context_set_heads.restype = _I
    L.bia_learned_head_eval.argtypes = [_V, _I, _I, _V, _V]
    L.bia_learned_head_eval.restype = _I
    L.bia_dim_integrate.argtypes = [_V, _I, _D, _V, _D, _D, _D, _D, ctypes.POINTER(BiaDimStats)]
    L.bia_dim_integrate.restype = _I
    _PI = ctypes.POINTER(ctypes.c_int)
    L.rkf_c_.argtypes = [_I, _D, _PD, _PD, _PD, _PI, _PD, _PD, _PD, _PD, _PI, _PI, _PD, _PD, _PD,
                         _PD, _PD]
    L.rkf_c_.restype = None
    L.find_dxyuv_kernel_.argtypes = [_I, _I, _I, _D, _D, _I] + [_PD] * 8
    L.find_dxyuv_kernel_.restype = None
    L.invariance_gpu_.argtypes = [_I, _D] + [_PD] * 6 + [_PD] * 11
    L.invariance_gpu_.restype = None
    _PF = ctypes.POINTER(ctypes.c_float)
    L.bia_trainer_create.argtypes = [_V, _I, ctypes.c_longlong, ctypes.c_ulonglong, ctypes.POINTER(_V)]
    L.bia_trainer_destroy.argtypes = [_V]
    L.bia_trainer_param_count.argtypes = []
    L.bia_trainer_get_params.argtypes = [_V, _PF]
    L.bia_trainer_set_params.argtypes = [_V, _PF]
    L.bia_trainer_gradient.argtypes = [_V, _V, _V, _I, _PF, _PF]
    L.bia_trainer_train.argtypes = [_V, _I, _I, ctypes.c_float, _PF]
    L.bia_trainer_export.argtypes = [_V, ctypes.c_char_p]
    L.bia_trainer_samples.argtypes = [_V, ctypes.POINTER(_V), ctypes.POINTER(_V),
                                      ctypes.POINTER(ctypes.c_longlong)]
    L.bia_trainer_copy_samples.argtypes = [_V, ctypes.c_longlong, ctypes.c_longlong, _PF, _PF]
    for name in ("bia_trainer_create", "bia_trainer_destroy", "bia_trainer_param_count",
                 "bia_trainer_get_params", "bia_trainer_set_params", "bia_trainer_gradient",
                 "bia_trainer_train", "bia_trainer_export", "bia_trainer_samples",
                 "bia_trainer_copy_samples"):
        getattr(L, name).restype = _I
    for name in ("bia_context_create", "bia_context_destroy", "bia_context_set_stream",
                 "bia_context_set_timing", "bia_context_kernel_ms", "bia_step", "bia_run",
                 "bia_run_host", "bia_invariance", "bia_measure_fp64_peak", "bia_context_stats"):
        getattr(L, name).restype = _I
    _lib = L
    return L


def status_string(status):
    try:
        return lib().bia_status_string(status).decode()
    except RuntimeError:
        return f"status {status}"


def check(status, what=""):
    if status != BIA_OK:
        raise BiaError(status, what)


def default_config(**overrides):
    cfg = BiaConfig()
    lib().bia_config_default(ctypes.byref(cfg))
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise AttributeError(f"bia_config has no field {k!r}")
        setattr(cfg, k, v)
    return cfg


EXPORTED_SYMBOLS = ("bia_config_default", "bia_context_create", "bia_context_destroy",
                    "bia_context_set_stream", "bia_context_set_timing", "bia_context_kernel_ms",
                    "bia_step", "bia_run", "bia_run_host", "bia_invariance", "bia_status_string",
                    "bia_measure_fp64_peak", "bia_context_stats", "bia_dim_integrate", "rkf_c_",
                    "bia_ensemble_create", "bia_ensemble_destroy", "bia_ensemble_particles",
                    "bia_ensemble_run", "bia_ensemble_energy", "bia_ensemble_autotune",
                    "bia_context_set_heads", "bia_learned_head_eval", "bia_context_autotune", "bia_context_set_shape",
                    "bia_selftest_wait_timeout", "bia_step_noalloc",
                    "bia_shard_columns", "bia_step_shard", "bia_apply_update",
                    "bia_trainer_create", "bia_trainer_destroy", "bia_trainer_param_count",
                    "bia_trainer_get_params", "bia_trainer_set_params", "bia_trainer_gradient",
                    "bia_trainer_train", "bia_trainer_export", "bia_trainer_samples",
                    "bia_trainer_copy_samples",
                    "bia_last_error", "find_dxyuv_kernel_", "invariance_gpu_")


def shard_columns(n, shard, nshards):
    """(c0, c1): the 32-particle column blocks whose pairs shard `shard` of `nshards` owns
    (host-only, no GPU needed)."""
    c0, c1 = ctypes.c_int(0), ctypes.c_int(0)
    check(lib().bia_shard_columns(int(n), int(shard), int(nshards), ctypes.byref(c0), ctypes.byref(c1)),
          "bia_shard_columns")
    return c0.value, c1.value
