"""ctypes binding of ``libstopeps_gpu.so`` (declared in ``include/stopeps_gpu.h``).

The library is required: importing the engine on a machine without the built
library, or calling it without a CUDA device, raises instead of falling back
to any CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libstopeps_gpu.so")

EXPORTS = [
    "sps_create", "sps_destroy", "sps_last_error", "sps_counters",
    "sps_identity_pepo", "sps_state_upload", "sps_state_layout", "sps_state_download",
    "sps_state_info", "sps_state_set_beta", "sps_state_copy", "sps_state_free",
    "sps_normalize_state", "sps_evolution_step", "sps_lognorm", "sps_measure_energy",
    "sps_set_truncated_svd", "sps_set_site_fields", "sps_set_variational", "sps_lognorm_variational", "sps_lognorm_gradient", "sps_lognorm_field_gradient", "sps_sampling_cache", "sps_sampling_cache_kind", "sps_sampling_cache_free", "sps_sample",
    "sps_sample_probability", "sps_sample_probability_batch",
    "sps_sample_batch", "sps_project", "sps_set_profile", "sps_kernel_stats_json", "sps_timer_start",
    "sps_timer_stop", "sps_la_svd", "sps_la_qr", "sps_la_svd_noalloc", "sps_la_svd_left", "sps_la_svd_topk", "sps_la_gemm", "sps_set_concurrency",
    "sps_set_sm_share", "sps_project_batch", "sps_evolution_step_batch", "sps_measure_energy_batch",
    "sps_lognorm_batch", "sps_set_injection", "sps_set_precision", "sps_la_gemm_mixed",
    "sps_set_autotune", "sps_autotune_report",
    "sps_sample_conditionals",
]

STATUS = {0: "SPS_OK", 1: "SPS_ERR_ARGUMENT", 2: "SPS_ERR_CUDA", 3: "SPS_ERR_NUMERIC",
          4: "SPS_ERR_BORN", 5: "SPS_ERR_CONVERGENCE", 6: "SPS_ERR_REPAIR", 7: "SPS_ERR_STATE"}


class sps_config(C.Structure):
    _fields_ = [("Lx", C.c_int32), ("Ly", C.c_int32), ("J", C.c_double), ("h", C.c_double),
                ("trotter_order", C.c_int32), ("fu_max_iterations", C.c_int32),
                ("fu_error_tolerance", C.c_double), ("fu_diagonal_shift", C.c_double),
                ("fu_linear_max_iterations", C.c_int32), ("fu_linear_tolerance", C.c_double),
                ("record_boundary_entropy", C.c_int32), ("device", C.c_int32)]


class sps_boundary(C.Structure):
    _fields_ = [("chi", C.c_int32), ("space0", C.c_int32), ("space1", C.c_int32), ("absorption", C.c_int32)]


class sps_step_report(C.Structure):
    _fields_ = [("beta", C.c_double), ("max_state_truncation", C.c_double),
                ("max_environment_truncation", C.c_double), ("max_boundary_entropy", C.c_double),
                ("max_solver_residual", C.c_double), ("max_iteration_limit_error", C.c_double),
                ("bond_updates", C.c_int32), ("iteration_limit_hits", C.c_int32),
                ("stop_error_tolerance", C.c_int32), ("stop_iteration_limit", C.c_int32),
                ("stop_residual_fallback", C.c_int32), ("stop_disabled", C.c_int32),
                ("linear_unconverged_updates", C.c_int32), ("repairs", C.c_int32),
                ("fallbacks", C.c_int32), ("log_normalization_sum", C.c_double)]


class sps_lognorm_result(C.Structure):
    _fields_ = [("log_norm", C.c_double), ("tensor_log_norm", C.c_double),
                ("max_environment_truncation", C.c_double)]


class sps_energy(C.Structure):
    _fields_ = [("energy_total", C.c_double), ("energy_per_site", C.c_double), ("log_norm", C.c_double),
                ("tensor_log_norm", C.c_double), ("max_environment_truncation", C.c_double),
                ("x_sum", C.c_double), ("zz_sum", C.c_double)]


class sps_sample_report(C.Structure):
    _fields_ = [("log_probability", C.c_double), ("max_environment_truncation", C.c_double),
                ("near_boundary", C.c_int32), ("metric_repairs", C.c_int32), ("zero_proposals", C.c_int32),
                ("min_relative_eigenvalue", C.c_double)]


_lib = None


def load():
    """Load the library once; raise if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise RuntimeError(f"{LIBPATH} is missing: build it with __graft_entry__.build()")
    lib = C.CDLL(LIBPATH)
    P = C.POINTER
    i32, i64, dbl, vp = C.c_int32, C.c_int64, C.c_double, C.c_void_p
    sig = {
        "sps_create": ([P(sps_config), P(vp)], C.c_int),
        "sps_destroy": ([vp], None),
        "sps_last_error": ([vp, C.c_char_p, C.c_size_t], C.c_int),
        "sps_counters": ([vp, P(C.c_longlong), P(dbl)], C.c_int),
        "sps_identity_pepo": ([vp, P(i32)], C.c_int),
        "sps_state_upload": ([vp, i32, dbl, dbl, P(i32), P(dbl), P(i32)], C.c_int),
        "sps_state_layout": ([vp, i32, P(i32), P(i64)], C.c_int),
        "sps_state_download": ([vp, i32, P(dbl), i64], C.c_int),
        "sps_state_info": ([vp, i32, P(dbl), P(dbl), P(i32)], C.c_int),
        "sps_state_set_beta": ([vp, i32, dbl], C.c_int),
        "sps_state_copy": ([vp, i32, P(i32)], C.c_int),
        "sps_state_free": ([vp, i32], C.c_int),
        "sps_normalize_state": ([vp, i32, P(dbl)], C.c_int),
        "sps_evolution_step": ([vp, i32, dbl, i32, P(i32), P(sps_boundary), P(sps_step_report)], C.c_int),
        "sps_lognorm": ([vp, i32, P(sps_boundary), P(sps_lognorm_result)], C.c_int),
        "sps_measure_energy": ([vp, i32, P(sps_boundary), P(sps_energy), P(dbl), P(dbl), P(dbl)], C.c_int),
        "sps_sampling_cache": ([vp, i32, P(sps_boundary), P(i32)], C.c_int),
        "sps_sampling_cache_free": ([vp, i32], C.c_int),
        "sps_sample": ([vp, i32, P(dbl), P(i32), P(sps_sample_report)], C.c_int),
        "sps_sample_probability": ([vp, i32, P(i32), P(sps_sample_report)], C.c_int),
        "sps_sample_probability_batch": ([vp, i32, i32, P(i32), P(dbl), P(sps_sample_report)], C.c_int),
        "sps_sampling_cache_kind": ([vp, i32, P(sps_boundary), i32, P(i32)], C.c_int),
        "sps_set_truncated_svd": ([vp, i32], C.c_int),
        "sps_set_site_fields": ([vp, i32, C.POINTER(C.c_double)], C.c_int),
        "sps_set_variational": ([vp, i32, C.c_double], C.c_int),
        "sps_lognorm_field_gradient": ([vp, i32, P(sps_boundary), i32, C.POINTER(C.c_double),
                                        C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
        "sps_lognorm_gradient": ([vp, i32, P(sps_boundary), i32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                  C.c_int64], C.c_int),
        "sps_lognorm_variational": ([vp, i32, C.POINTER(sps_boundary), C.POINTER(sps_lognorm_result),
                                     C.POINTER(C.c_int32), C.POINTER(C.c_double)], C.c_int),
        "sps_sample_conditionals": ([vp, i32, P(dbl), P(i32), P(i32), P(dbl), P(sps_sample_report)], C.c_int),
        "sps_sample_batch": ([vp, i32, i32, P(dbl), P(i32), P(dbl), P(sps_sample_report)], C.c_int),
        "sps_project": ([vp, i32, P(i32), P(i32), P(dbl)], C.c_int),
        "sps_project_batch": ([vp, i32, i32, P(i32), P(i32), P(dbl)], C.c_int),
        "sps_evolution_step_batch": ([vp, i32, P(i32), P(dbl), i32, P(i32), P(sps_boundary), P(sps_step_report)],
                                     C.c_int),
        "sps_measure_energy_batch": ([vp, i32, P(i32), P(sps_boundary), P(sps_energy), P(dbl)], C.c_int),
        "sps_lognorm_batch": ([vp, i32, P(i32), P(sps_boundary), P(sps_lognorm_result)], C.c_int),
        "sps_set_profile": ([vp, i32], C.c_int),
        "sps_set_injection": ([vp, i32, i32, i32], C.c_int),
        "sps_set_precision": ([vp, i32], C.c_int),
        "sps_set_autotune": ([vp, i32], C.c_int),
        "sps_autotune_report": ([vp, C.c_char_p, C.c_size_t], C.c_int),
        "sps_la_gemm_mixed": ([vp, i32, i32, i32, i32, P(dbl), P(dbl), P(dbl), P(dbl)], C.c_int),
        "sps_kernel_stats_json": ([vp, C.c_char_p, C.c_size_t], C.c_int),
        "sps_timer_start": ([vp], C.c_int),
        "sps_timer_stop": ([vp, P(dbl)], C.c_int),
        "sps_la_svd": ([vp, i32, i32, P(dbl), P(dbl), P(dbl), P(dbl), P(i32), P(dbl)], C.c_int),
        "sps_la_qr": ([vp, i32, i32, P(dbl), P(dbl), P(dbl), P(dbl)], C.c_int),
        "sps_la_svd_noalloc": ([i32, vp, i32, i32, vp, vp, vp, vp], C.c_int),
        "sps_la_svd_left": ([vp, i32, i32, P(dbl), P(dbl), P(dbl), P(i32), P(dbl)], C.c_int),
        "sps_set_concurrency": ([vp, i32], C.c_int),
        "sps_set_sm_share": ([vp, i32], C.c_int),
        "sps_la_gemm": ([vp, i32, i32, i32, i32, dbl, P(dbl), P(dbl), dbl, P(dbl), P(dbl)], C.c_int),
        "sps_la_svd_topk": ([vp, i32, i32, i32, P(dbl), i32, C.c_double, P(dbl), P(dbl), P(dbl), P(i32), P(dbl)],
                            C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


class EngineError(RuntimeError):
    def __init__(self, code, message):
        super().__init__(f"{STATUS.get(code, code)}: {message}")
        self.code = code
