"""ctypes binding of libmgkmc_b200.so (the C ABI in include/mgkmc_b200.h).

There is no fallback: if the native library is missing or no CUDA device is
present, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmgkmc_b200.so")

STATUS = {0: "MGK_OK", 1: "MGK_LS_NOT_CONVERGED", 2: "MGK_BAD_SHAPE", 3: "MGK_OOM", 4: "MGK_DEVICE_TIMEOUT",
          5: "MGK_CUDA_ERROR", 6: "MGK_BAD_ARG", 7: "MGK_UNSUPPORTED", 8: "MGK_TERMINATED",
          9: "MGK_TIME_LIMIT"}

EXPORTS = ["mgk_last_error", "mgk_version", "mgk_device_count", "mgk_ls_create", "mgk_ls_solve", "mgk_ls_destroy",
           "mgk_kmc_create", "mgk_kmc_run", "mgk_kmc_elastic_run", "mgk_kmc_get_field", "mgk_kmc_get_macro",
           "mgk_kmc_destroy", "mgk_kmc_set_profiling", "mgk_kmc_get_profile", "mgk_batch_create", "mgk_batch_run",
           "mgk_batch_stats", "mgk_batch_get_field", "mgk_batch_get_macro", "mgk_batch_set_time_limit", "mgk_batch_event_times", "mgk_le_run",
           "mgk_batch_create_from", "mgk_device_memory", "mgk_correlated_field",
           "mgk_ls_set_precision", "mgk_ls_last_solve_ms", "mgk_ls_set_wait_limit", "mgk_ls_inject_absent_cta", "mgk_ls_plan", "mgk_set_batch_plan",
           "mgk_get_device", "mgk_set_device", "mgk_batch_destroy"]


class MgkError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__("%s: %s" % (STATUS.get(status, str(status)), msg))
        self.status = status


class KmcParamsC(C.Structure):
    _fields_ = [("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("M", C.c_int),
                ("plane_stress", C.c_int), ("seed", C.c_int), ("gamma0", C.c_double), ("pixel", C.c_double),
                ("barrier_type", C.c_int), ("bar_mean", C.c_double), ("bar_std", C.c_double),
                ("bar_min_cutoff", C.c_double), ("bar_max_cutoff", C.c_double), ("bar_loc", C.c_double),
                ("bar_scale", C.c_double), ("bar_epsilon", C.c_double), ("bar_ratio", C.c_double),
                ("directional", C.c_int), ("softening_cap", C.c_double), ("jp", C.c_double), ("jt", C.c_double),
                ("neighbor_fraction", C.c_double), ("q_act_temp", C.c_double), ("temperature", C.c_double),
                ("strain_rate", C.c_double), ("stability_threshold", C.c_double), ("nu0", C.c_double),
                ("instability_kmc", C.c_int), ("scale_rate_by_volume", C.c_int), ("redraw_directions", C.c_int),
                ("redraw_barriers", C.c_int), ("use_3d_barriers", C.c_int), ("fast_patching", C.c_int),
                ("patch_radius", C.c_int), ("sync_interval", C.c_int), ("ls_tol", C.c_double),
                ("ls_max_iter", C.c_int), ("catalog_type", C.c_int), ("barrier_per_voxel", C.c_int),
                ("ls_precision", C.c_int)]


class LeParamsC(C.Structure):
    _fields_ = [("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("plane_stress", C.c_int),
                ("pixel", C.c_double), ("eps_target", C.c_double), ("step_size", C.c_double), ("drive_i", C.c_int),
                ("drive_j", C.c_int), ("n_targets", C.c_int), ("target_i", C.c_int * 9), ("target_j", C.c_int * 9),
                ("target_v", C.c_double * 9), ("mixed_tol", C.c_double), ("max_iter_macro", C.c_int),
                ("max_iter_ls", C.c_int), ("tol_ls", C.c_double), ("output_dir", C.c_char_p),
                ("summary_filename", C.c_char_p), ("enable_summary_log", C.c_int), ("enable_global_log", C.c_int),
                ("enable_console", C.c_int), ("vtk_interval", C.c_char_p)]


class RunParamsC(C.Structure):
    _fields_ = [("n_global_steps", C.c_int), ("step_size", C.c_double), ("comp_i", C.c_int), ("comp_j", C.c_int),
                ("n_targets", C.c_int), ("target_i", C.c_int * 9), ("target_j", C.c_int * 9),
                ("target_v", C.c_double * 9), ("mixed_tol", C.c_double), ("mixed_max_iter", C.c_int),
                ("max_kmc_steps_pct", C.c_double), ("max_events", C.c_longlong), ("output_dir", C.c_char_p),
                ("summary_filename", C.c_char_p), ("enable_summary_log", C.c_int), ("enable_global_log", C.c_int),
                ("enable_console", C.c_int), ("vtk_interval", C.c_char_p), ("vtk_elastic_only", C.c_int),
                ("max_cascade_batches", C.c_longlong)]


_lib = None


def lib():
    """Load the native library (built by mgkmc_cpp_b200/build.py)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("native library missing: %s (run `python -m mgkmc_cpp_b200.build`)" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    dp = C.POINTER(C.c_double)
    vp = C.c_void_p
    L.mgk_last_error.restype = C.c_char_p
    L.mgk_version.restype = C.c_int
    L.mgk_device_count.restype = C.c_int
    L.mgk_ls_create.argtypes = [C.POINTER(vp), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, dp, dp]
    L.mgk_ls_solve.argtypes = [vp, dp, dp, dp, C.c_int, dp, dp, C.c_int, C.c_double, C.POINTER(C.c_int)]
    L.mgk_ls_destroy.argtypes = [vp]
    L.mgk_ls_destroy.restype = None
    L.mgk_kmc_create.argtypes = [C.POINTER(vp), C.POINTER(KmcParamsC), dp, dp]
    L.mgk_kmc_run.argtypes = [vp, C.POINTER(RunParamsC), dp, C.c_longlong, C.POINTER(C.c_longlong)]
    L.mgk_kmc_elastic_run.argtypes = [vp]
    L.mgk_kmc_get_field.argtypes = [vp, C.c_int, dp, C.POINTER(C.c_longlong)]
    L.mgk_kmc_get_macro.argtypes = [vp, dp, C.c_int]
    L.mgk_kmc_set_profiling.argtypes = [vp, C.c_int]
    L.mgk_kmc_get_profile.argtypes = [vp, dp, dp, C.c_longlong]
    L.mgk_batch_create.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(KmcParamsC), C.POINTER(dp), C.POINTER(dp)]
    L.mgk_batch_run.argtypes = [vp, C.POINTER(RunParamsC), C.c_longlong, dp]
    L.mgk_batch_stats.argtypes = [vp, C.c_int, dp, C.POINTER(C.c_int), C.c_longlong, C.POINTER(C.c_longlong)]
    L.mgk_batch_get_field.argtypes = [vp, C.c_int, C.c_int, dp, C.POINTER(C.c_longlong)]
    L.mgk_batch_get_macro.argtypes = [vp, C.c_int, dp, C.c_int]
    L.mgk_batch_set_time_limit.argtypes = [vp, C.c_double]
    L.mgk_batch_create_from.argtypes = [C.POINTER(vp), C.c_int, C.POINTER(vp)]
    L.mgk_device_memory.argtypes = [C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]
    L.mgk_correlated_field.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                       C.c_double, C.c_int, C.c_double, C.c_int, dp]
    L.mgk_ls_set_precision.argtypes = [vp, C.c_int]
    L.mgk_ls_last_solve_ms.argtypes = [vp, dp]
    L.mgk_ls_set_wait_limit.argtypes = [vp, C.c_double]
    L.mgk_ls_inject_absent_cta.argtypes = [vp, C.c_int]
    L.mgk_ls_plan.argtypes = [vp, C.POINTER(C.c_int)]
    L.mgk_set_batch_plan.argtypes = [C.c_int]
    L.mgk_get_device.argtypes = [C.POINTER(C.c_int)]
    L.mgk_set_device.argtypes = [C.c_int]
    L.mgk_le_run.argtypes = [C.POINTER(LeParamsC), dp, dp, dp, C.POINTER(C.c_int)]
    L.mgk_batch_event_times.argtypes = [vp, C.c_int, dp, C.c_longlong, C.POINTER(C.c_longlong)]
    L.mgk_batch_destroy.argtypes = [vp]
    L.mgk_batch_destroy.restype = None
    L.mgk_kmc_destroy.argtypes = [vp]
    L.mgk_kmc_destroy.restype = None
    for fn in ("mgk_ls_create", "mgk_ls_solve", "mgk_kmc_create", "mgk_kmc_run", "mgk_kmc_elastic_run",
               "mgk_kmc_get_field", "mgk_kmc_get_macro", "mgk_kmc_set_profiling", "mgk_kmc_get_profile",
               "mgk_batch_create", "mgk_batch_run", "mgk_batch_stats", "mgk_batch_get_field", "mgk_batch_get_macro",
               "mgk_batch_set_time_limit", "mgk_batch_event_times", "mgk_le_run",
               "mgk_batch_create_from", "mgk_device_memory", "mgk_correlated_field",
               "mgk_ls_set_precision", "mgk_ls_last_solve_ms", "mgk_ls_set_wait_limit", "mgk_ls_inject_absent_cta", "mgk_ls_plan", "mgk_set_batch_plan",
               "mgk_get_device", "mgk_set_device"):
        getattr(L, fn).restype = C.c_int
    _lib = L
    return L


def check(status: int, allow=()) -> int:
    if status != 0 and status not in allow:
        raise MgkError(status, lib().mgk_last_error().decode(errors="replace"))
    return status


def require_device():
    if lib().mgk_device_count() < 1:
        raise MgkError(5, "no CUDA device visible to libmgkmc_b200")


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None
