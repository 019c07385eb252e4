"""ctypes binding of libjfdk.so (include/jfdk.h).

Loading fails loudly when the library is missing: the engine has no CPU
fallback.  Build it with ``python -m jenhine_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libjfdk.so")

JFDK_OK = 0
JFDK_ERR_INVALID = -1
JFDK_ERR_CUDA = -2
JFDK_ERR_OOM = -3
JFDK_ERR_UNSUPPORTED = -4
JFDK_ERR_STATE = -5
JFDK_ERR_NO_DEVICE = -6

PRECISION_FP32 = 0
PRECISION_MIXED = 1

OPT_BP_EXACT = 1
OPT_VIEW_CHUNK = 2
OPT_STAGE_TIMING = 3
OPT_BP_ZPT = 4
OPT_FILTER_SIMT = 5
OPT_RAMP_PRODUCT = 6
OPT_DEVICE_MEMORY_LIMIT = 7
OPT_BP_TILE = 8
OPT_BP_WEIGHTS = 9
AUTOTUNE_FORCE = 1
BATCH_AUTOTUNE, BATCH_GRAPH, BATCH_PERSISTENT, BATCH_PIPELINED = 1, 2, 4, 8
RAMP_DEFAULT, RAMP_TF32X3, RAMP_BF16X3, RAMP_FP16X3, RAMP_FP32_SIMT, RAMP_I8X14 = 0, 1, 2, 3, 4, 5


class ScanParams(C.Structure):
    """Config/ScanParams.h:13-40."""
    _fields_ = [
        ("num_views", C.c_int), ("dso", C.c_float), ("dsd", C.c_float),
        ("num_dets_u", C.c_int), ("num_dets_v", C.c_int), ("detector_pixel_size", C.c_float),
        ("border_up", C.c_int), ("border_down", C.c_int), ("border_left", C.c_int),
        ("border_right", C.c_int), ("bright_field", C.c_float),
        ("beam_hardening", C.c_float * 3), ("half_sample_rate", C.c_float),
        ("detector_on_right", C.c_int), ("filter_input_width", C.c_int),
    ]


class ReconParams(C.Structure):
    """Config/ReconParams.h:14-68."""
    _fields_ = [
        ("num_pixels_x", C.c_int), ("num_pixels_y", C.c_int), ("num_pixels_z", C.c_int),
        ("pitch_xy", C.c_float), ("pitch_z", C.c_float), ("ct_norm0", C.c_float),
        ("ct_norm1", C.c_float), ("mu_water", C.c_float), ("filter_cutoff_start", C.c_float),
        ("filter_cutoff_end", C.c_float), ("num_adjust", C.c_int),
        ("adjust_points", C.POINTER(C.c_float)), ("adjust_level_db", C.POINTER(C.c_float)),
        ("z_filter", C.c_int),
    ]


class JfdkError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"jfdk status {status}: {msg}")
        self.status = status


_lib = None

# name -> (argtypes, restype)
_P = C.c_void_p
_SIGS = {
    "jfdk_create": ([C.POINTER(_P), C.POINTER(ScanParams), C.POINTER(ReconParams), _P, C.c_int, _P], C.c_int),
    "jfdk_destroy": ([_P], None),
    "jfdk_last_error": ([_P], C.c_char_p),
    "jfdk_sync": ([_P], C.c_int),
    "jfdk_get_dims": ([_P, _P, _P, _P, _P], C.c_int),
    "jfdk_set_option": ([_P, C.c_int, C.c_longlong], C.c_int),
    "jfdk_get_option": ([_P, C.c_int, C.POINTER(C.c_longlong)], C.c_int),
    "jfdk_stage_times": ([_P, _P], C.c_int),
    "jfdk_preprocess_frames": ([_P, _P, C.c_int, _P], C.c_int),
    "jfdk_filter_frames": ([_P, _P, C.c_int, C.c_int, _P], C.c_int),
    "jfdk_filter_frames_noalloc": ([_P, _P, C.c_int, C.c_int, _P], C.c_int),
    "jfdk_zfilter_frames": ([_P, _P, C.c_int], C.c_int),
    "jfdk_composite_frames": ([_P, _P, _P, C.c_int, C.c_int, _P], C.c_int),
    "jfdk_bp_reset": ([_P], C.c_int),
    "jfdk_bp_set_slab": ([_P, C.c_int, C.c_int], C.c_int),
    "jfdk_bp_reserve": ([_P, C.c_int], C.c_int),
    "jfdk_bp_accumulate": ([_P, _P, C.c_int, C.c_int], C.c_int),
    "jfdk_finalize": ([_P, C.c_int, C.c_int, C.c_int, _P, _P], C.c_int),
    "jfdk_ctnum": ([_P, _P, C.c_size_t], C.c_int),
    "jfdk_reconstruct": ([_P, _P, _P, _P], C.c_int),
    "jfdk_reconstruct_host": ([_P, _P, _P], C.c_int),
    "jfdk_get_uweights": ([_P, _P], C.c_int),
    "jfdk_get_ramp_operator": ([_P, _P, _P], C.c_int),
    "jfdk_kernel_launches": ([_P], C.c_longlong),
    "jfdk_device_bytes": ([_P], C.c_longlong),
    "jfdk_device_check": ([C.c_char_p, C.c_int], C.c_int),
    "jfdk_set_bp_geometry": ([_P, _P], C.c_int),
    "jfdk_bp_adjoint": ([_P, _P, C.c_int, C.c_int, _P], C.c_int),
    "jfdk_filter_adjoint": ([_P, _P, C.c_int, C.c_int, _P], C.c_int),
    "jfdk_geometry_gradient": ([_P, _P, C.c_int, C.c_int, _P, _P, _P, _P], C.c_int),
    "jfdk_autotune": ([_P, C.c_int], C.c_int),
    "jfdk_filter_to_store": ([_P, _P, C.c_int, C.c_int], C.c_int),
    "jfdk_filter_raw": ([_P, _P, C.c_int, C.c_int, _P], C.c_int),
    "jfdk_store_range": ([_P, C.c_int, C.c_int, _P, _P, _P], C.c_int),
    "jfdk_backproject_store": ([_P, C.c_int, C.c_int, _P, _P], C.c_int),
    "jfdk_batch_create": ([C.POINTER(_P), _P, C.c_int, C.c_int, _P], C.c_int),
    "jfdk_batch_destroy": ([_P], None),
    "jfdk_batch_last_error": ([_P], C.c_char_p),
    "jfdk_batch_run": ([_P, _P, _P], C.c_int),
    "jfdk_batch_launches": ([_P], C.c_longlong),
    "jfdk_batch_schedule": ([_P], C.c_int),
    "jfdk_measure_gather_rate": ([C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double)], C.c_int),
}


def exported_symbols():
    return sorted(_SIGS)


def load():
    """Load libjfdk.so once; raise if it is missing or incomplete."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `python -m jenhine_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(ctx, status: int) -> None:
    if status != JFDK_OK:
        msg = load().jfdk_last_error(ctx).decode() if ctx else ""
        raise JfdkError(status, msg)
