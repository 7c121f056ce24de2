"""ctypes binding of libsplat_b200.so (C ABI: include/splat_b200.h).

The library is the compute path; there is no fallback.  ``lib()`` raises
when the built library is missing or cannot be loaded.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# SPLAT_B200_LIB: load a library built elsewhere (default: the in-tree build)
LIB_PATH = os.environ.get("SPLAT_B200_LIB") or os.path.join(PKG_DIR, "libsplat_b200.so")
HEADER = os.path.join(os.path.dirname(PKG_DIR), "include", "splat_b200.h")

GS_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of device memory", -4: "device status fault",
          -5: "size limit exceeded"}


class GsOptions(C.Structure):
    _fields_ = [("eCut", C.c_float), ("aMin", C.c_float), ("radClamp", C.c_float), ("anisoReg", C.c_float),
                ("shDeg", C.c_int32), ("tileGrad", C.c_int32), ("entriesCap", C.c_uint64),
                ("maxSplats", C.c_uint32), ("maxIters", C.c_uint32), ("capMult", C.c_double),
                ("minScale", C.c_double), ("growRate", C.c_double), ("growUntil", C.c_double),
                ("opacityReg", C.c_float), ("shLr", C.c_float), ("tile", C.c_int32), ("batchDepth", C.c_int32),
                ("maxBatch", C.c_int32), ("backwardVariant", C.c_int32), ("persistent", C.c_int32),
                ("useGraphs", C.c_int32), ("device", C.c_int32), ("tileCull", C.c_int32),
                ("donorSampling", C.c_int32)]


class GsCamera(C.Structure):
    _fields_ = [("R", C.c_float * 9), ("t", C.c_float * 3), ("f", C.c_float), ("cx", C.c_float),
                ("cy", C.c_float), ("w", C.c_int32), ("h", C.c_int32), ("imgIdx", C.c_int32), ("g", C.c_double),
                ("b", C.c_double)]


class GsImage(C.Structure):
    _fields_ = [("tw", C.c_uint32), ("th", C.c_uint32), ("rgb", C.POINTER(C.c_float))]


class GsFrame(C.Structure):
    _fields_ = [("tw", C.c_uint32), ("th", C.c_uint32), ("fw", C.c_double), ("rgb", C.POINTER(C.c_float))]


GS_E_LIMIT = -5
STATIC_SORT_MAX = 1 << 20  # GS_STATIC_SORT_MAX of include/splat_b200.h


class GsState(C.Structure):
    _fields_ = [("iter", C.c_uint32), ("n", C.c_uint32), ("cap", C.c_uint32), ("shDeg", C.c_uint32),
                ("shK", C.c_uint32), ("stride", C.c_uint32), ("ncams", C.c_uint32), ("maxTiles", C.c_uint32),
                ("pixelsSeen", C.c_uint64), ("entriesCap", C.c_uint64), ("horizon", C.c_uint32),
                ("lastEntries", C.c_uint32), ("stepUploadBytes", C.c_uint32),
                ("lastLaunches", C.c_uint32)]


class GsRefineResult(C.Structure):
    _fields_ = [("moved", C.c_uint32), ("grown", C.c_uint32), ("n", C.c_uint32), ("maxTile", C.c_uint32),
                ("overflow", C.c_uint32), ("early", C.c_int32)]


RNG_FN = C.CFUNCTYPE(C.c_double, C.c_void_p)

_lib = None


def lib():
    """Load the CUDA library (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built (run splat.js_b200/build.py); there is no CPU fallback")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    H = C.c_void_p
    f32p, u32p, i32p, u64p = P(C.c_float), P(C.c_uint32), P(C.c_int32), P(C.c_uint64)
    sig = {
        "gs_abi_version": (C.c_int, []),
        "gs_default_options": (C.c_int, [P(GsOptions)]),
        "gs_create": (C.c_int, [P(GsOptions), P(H)]),
        "gs_destroy": (None, [H]),
        "gs_last_error": (C.c_char_p, [H]),
        "gs_setup": (C.c_int, [H, f32p, C.c_uint32, f32p, P(GsCamera), C.c_uint32, P(GsImage), C.c_uint32,
                               C.c_uint32, C.c_uint32, C.c_double]),
        "gs_get_state": (C.c_int, [H, P(GsState)]),
        "gs_set_iter": (C.c_int, [H, C.c_uint32]),
        "gs_set_horizon": (C.c_int, [H, C.c_uint32]),
        "gs_set_grow_limit": (C.c_int, [H, C.c_uint32]),
        "gs_set_camera": (C.c_int, [H, C.c_uint32, P(GsCamera)]),
        "gs_step": (C.c_int, [H, C.c_uint32]),
        "gs_step_batch": (C.c_int, [H, u32p, C.c_uint32]),
        "gs_read_stats": (C.c_int, [H, u32p]),
        "gs_read_stats_async": (C.c_int, [H, C.c_void_p]),
        "gs_read_gaussians": (C.c_int, [H, f32p, f32p, u32p]),
        "gs_export_ply": (C.c_int, [H, C.c_int32, C.c_double, P(C.c_double), C.c_uint32, C.c_void_p, C.c_uint64,
                                    u64p]),
        "gs_write_gaussians": (C.c_int, [H, f32p, f32p, C.c_uint32]),
        "gs_read_moments": (C.c_int, [H, f32p, f32p, f32p, f32p]),
        "gs_reset_moments": (C.c_int, [H]),
        "gs_render": (C.c_int, [H, P(GsCamera), C.c_int32, C.c_uint32, f32p]),
        "gs_eval_pass": (C.c_int, [H, C.c_uint32, P(GsCamera), u32p, i32p]),
        "gs_grad_pass": (C.c_int, [H, C.c_uint32, f32p, f32p, u32p]),
        "gs_read_cam_grads": (C.c_int, [H, i32p, C.c_int32]),
        "gs_refine": (C.c_int, [H, RNG_FN, C.c_void_p, P(GsRefineResult)]),
        "gs_sync": (C.c_int, [H]),
        "gs_set_stream": (C.c_int, [H, C.c_void_p]),
        "gs_profile": (C.c_int, [H, C.c_int32]),
        "gs_profile_read": (C.c_int, [H, P(C.c_double), u32p]),
        "gs_probe_fp32_peak": (C.c_int, [C.c_int32, P(C.c_double)]),
        "gs_debug_check_rcp": (C.c_int, [C.c_int32, u64p, u32p]),
        "gs_sort_entries_static": (C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]),
        "gs_autotune": (C.c_int, [H, u32p, C.c_uint32, C.c_int32, i32p, i32p, f32p]),
        "gs_set_raster_config": (C.c_int, [H, C.c_int32, C.c_int32]),
        "gs_set_tile_cull": (C.c_int, [H, C.c_int32]),
        "gs_raster_pass": (C.c_int, [H, u32p, C.c_uint32, C.c_int32]),
        "gs_debug_records": (C.c_int, [H, C.c_uint32, f32p, u32p]),
        "gs_debug_binning": (C.c_int, [H, C.c_uint32, u32p, u32p, u32p, C.c_uint64, u64p]),
        "gs_debug_pixels": (C.c_int, [H, C.c_uint32, f32p, f32p, u32p]),
        "gs_debug_lookback_timeout": (C.c_int, [C.c_int32, C.c_uint32, u32p, P(C.c_double)]),
        "gs_debug_gradp": (C.c_int, [H, C.c_uint32, i32p, C.c_int32]),
        "gs_undistort_frames": (C.c_int, [C.c_int32, P(GsFrame), C.c_uint32, C.c_double, C.c_double, C.c_double,
                                          i32p]),
        "gs_debug_targets": (C.c_int, [H, u32p, C.c_uint64]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def ptr(a, ct=C.c_float):
    """Pointer to a contiguous numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ct))


class GSError(RuntimeError):
    pass


def check(rc, handle=None):
    if rc != GS_OK:
        msg = lib().gs_last_error(handle)
        raise GSError(f"{ERRORS.get(rc, rc)}: {msg.decode() if msg else ''}")
