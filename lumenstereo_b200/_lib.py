"""ctypes binding of liblumen_sgbm.so (the C ABI in include/lumen_sgbm.h).

The shared library is built in-tree by ``lumenstereo_b200.build``.  There is no
CPU or Python fallback: if the library cannot be loaded, every entry point
raises, so a GPU run can never silently measure something else.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblumen_sgbm.so")

_lock = threading.Lock()
_lib = None

# lumen_status
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_RANGE_EXCEEDS_LIMIT = 2
ERR_CUDA = 3
ERR_OUT_OF_BUDGET = 4
ERR_TIMEOUT = 5
ERR_NO_DEVICE = 6

PARAM_FIELDS = ("minDisparity", "maxDisparity", "blockSize", "P1", "P2", "preFilterCap",
                "uniquenessRatio", "disp12MaxDiff", "speckleWindowSize", "speckleRange",
                "useGPU", "useSharedMemory", "numDirections", "matchingCostMode")


class CParams(C.Structure):
    _fields_ = [(n, C.c_int32) for n in PARAM_FIELDS]


class CServerOptions(C.Structure):
    _fields_ = [("device_budget_bytes", C.c_size_t), ("max_batch_pairs", C.c_int),
                ("rows_per_band", C.c_int), ("max_inflight", C.c_int), ("watchdog_ms", C.c_int),
                ("spin_limit", C.c_longlong), ("plain_fallback", C.c_int), ("schedule", C.c_int)]


class CRequestInfo(C.Structure):
    _fields_ = [("status", C.c_int), ("latency_ms", C.c_double), ("queue_ms", C.c_double),
                ("device_ms", C.c_double), ("batch_pairs", C.c_int), ("batch_id", C.c_ulonglong)]


class CServerStats(C.Structure):
    _fields_ = [(n, C.c_ulonglong) for n in ("submitted", "completed", "rejected", "failed", "batches",
                                              "watchdog_expired")] + \
               [(n, C.c_size_t) for n in ("budget_bytes", "admitted_bytes", "peak_admitted_bytes")] + \
               [(n, C.c_int) for n in ("queue_depth", "peak_queue_depth", "inflight_batches",
                                       "peak_batch_pairs")] + \
               [("fallbacks", C.c_ulonglong)]


def _declare(lib):
    vp, i, sz = C.c_void_p, C.c_int, C.c_size_t
    sig = {
        "lumen_stereo_params_default": (None, [C.POINTER(CParams)]),
        "lumen_stereo_params_is_valid": (i, [C.POINTER(CParams)]),
        "lumen_stereo_params_auto_penalties": (None, [C.POINTER(CParams), i]),
        "lumen_sgbm_create": (i, [C.POINTER(CParams), C.POINTER(vp)]),
        "lumen_sgbm_destroy": (i, [vp]),
        "lumen_sgbm_set_params": (i, [vp, C.POINTER(CParams)]),
        "lumen_sgbm_get_params": (i, [vp, C.POINTER(CParams)]),
        "lumen_sgbm_compute": (i, [vp, vp, vp, i, i, sz, i, vp, sz]),
        "lumen_sgbm_compute_device": (i, [vp, vp, vp, i, i, sz, i, vp, sz, vp]),
        "lumen_sgbm_get_timings": (i, [vp, C.POINTER(C.c_float)]),
        "lumen_last_error_string": (C.c_char_p, []),
        "lumen_sgbm_debug_set_paths": (i, [vp, C.c_uint32]),
        "lumen_sgbm_set_schedule": (i, [vp, i]),
        "lumen_sgbm_set_tuning": (i, [vp, i, i]),
        "lumen_sgbm_set_tuning_columns": (i, [vp, i]),
        "lumen_sgbm_get_tuning_columns": (i, [vp, C.POINTER(C.c_int)]),
        "lumen_sgbm_debug_set_wait_limit": (i, [vp, C.c_longlong]),
        "lumen_sgbm_debug_stall_test": (i, [vp, i]),
        "lumen_sgbm_get_tuning": (i, [vp, C.POINTER(C.c_int)]),
        "lumen_sgbm_autotune": (i, [vp, vp, vp, i, i, sz, i, i, C.c_char_p, sz]),
        "lumen_sgbm_tuning_save": (i, [vp, C.c_char_p]),
        "lumen_sgbm_tuning_load": (i, [vp, C.c_char_p]),
        "lumen_sgbm_debug_retain": (i, [vp, i]),
        "lumen_sgbm_debug_copy": (i, [vp, i, vp, sz]),
        "lumen_sgbm_debug_launch_count": (C.c_ulonglong, [vp]),
        "lumen_sgbm_debug_trace": (i, [vp, i]),
        "lumen_sgbm_debug_trace_copy": (i, [vp, vp, sz, C.POINTER(sz)]),
        "lumen_rectifier_create": (i, [i, i, vp, vp, vp, vp, C.POINTER(vp)]),
        "lumen_rectifier_destroy": (i, [vp]),
        "lumen_rectifier_is_pre_rectified": (i, [vp]),
        "lumen_rectifier_rectify": (i, [vp, vp, vp, i, vp, vp]),
        "lumen_rectifier_rectify_device": (i, [vp, vp, vp, i, vp, vp, vp]),
        "lumen_remap": (i, [vp, vp, vp, vp, i, i, i]),
        "lumen_bgr_to_gray": (i, [vp, sz, vp, i, i]),
        "lumen_sgbm_batch_create": (i, [C.POINTER(vp)]),
        "lumen_sgbm_batch_destroy": (i, [vp]),
        "lumen_sgbm_batch_add": (i, [vp, C.POINTER(CParams), vp, vp, i, i, vp]),
        "lumen_sgbm_batch_clear": (i, [vp]),
        "lumen_sgbm_batch_set_options": (i, [vp, i, i, sz]),
        "lumen_sgbm_batch_run": (i, [vp, vp]),
        "lumen_sgbm_batch_sync": (i, [vp, vp]),
        "lumen_sgbm_batch_autotune": (i, [vp, vp, i, C.POINTER(C.c_int), C.POINTER(C.c_float)]),
        "lumen_sgbm_batch_info": (i, [vp, C.POINTER(sz), C.POINTER(C.c_int), C.POINTER(C.c_ulonglong)]),
        "lumen_sgbm_batch_set_schedule": (i, [vp, i]),
        "lumen_sgbm_batch_config": (i, [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "lumen_server_options_default": (None, [C.POINTER(CServerOptions)]),
        "lumen_server_create": (i, [C.POINTER(CServerOptions), C.POINTER(vp)]),
        "lumen_server_destroy": (i, [vp]),
        "lumen_server_set_calibration": (i, [vp, i, i, i, vp, vp, vp, vp]),
        "lumen_server_set_calibration_params": (i, [vp, i, i, i] + [vp] * 8),
        "lumen_server_submit": (i, [vp, C.POINTER(CParams), i, vp, vp, i, i, vp, C.POINTER(C.c_ulonglong)]),
        "lumen_server_wait": (i, [vp, C.c_ulonglong, i, C.POINTER(CRequestInfo)]),
        "lumen_server_get_stats": (i, [vp, C.POINTER(CServerStats)]),
        "lumen_server_debug_fail_batches": (i, [vp, i]),
        "lumen_debug_op_rates": (i, [C.POINTER(C.c_float)]),
        "lumen_disparity_to_depth_device": (i, [vp, i, i, sz, C.c_float, C.c_float, C.c_float, vp, sz, vp]),
        "lumen_rectify_maps_device": (i, [vp, vp, vp, vp, i, i, vp, vp, vp]),
        "lumen_disparity_to_depth_color_device": (i, [vp, i, i, sz, C.c_float, C.c_float, C.c_float, vp, sz,
                                                      C.c_float, C.c_float, vp, vp, sz, vp]),
        "lumen_depth_colorize_device": (i, [vp, i, i, sz, C.c_float, C.c_float, vp, vp, sz, vp]),
        "lumen_depth_to_points_device": (i, [vp, i, i, sz, vp, sz, C.c_double, C.c_double, C.c_double,
                                             C.c_double, vp, vp, vp]),
        "lumen_depth_to_points": (i, [vp, i, i, sz, vp, sz, C.c_double, C.c_double, C.c_double, C.c_double, vp,
                                      C.POINTER(C.c_int)]),
        "lumen_census_cost_noalloc": (i, [vp, vp, i, i, i, i, vp, i, vp]),
        "lumen_census_cost_noalloc_max_pixels": (sz, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def lib():
    """The loaded library (raises OSError when it is missing or unloadable)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not os.path.exists(LIB_PATH):
                    raise OSError(
                        f"{LIB_PATH} is missing: build it with `python -m lumenstereo_b200.build`")
                handle = C.CDLL(LIB_PATH)
                _declare(handle)
                _lib = handle
    return _lib


def last_error() -> str:
    msg = lib().lumen_last_error_string()
    return msg.decode() if msg else ""
