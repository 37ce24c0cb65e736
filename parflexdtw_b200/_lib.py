"""ctypes binding of the C ABI in ``include/parflexdtw_b200.h``.

The shared library is built in-tree (``python -m parflexdtw_b200.build``).
There is no CPU fallback: if the library is missing or no CUDA device is
present, every entry point raises.
"""
from __future__ import annotations

import ctypes as ct
import os
import threading

from . import build as _build

_i64 = ct.c_int64
_i32 = ct.c_int32
_f64 = ct.c_double
_vp = ct.c_void_p
_i64p = ct.POINTER(ct.c_int64)
_i32p = ct.POINTER(ct.c_int32)
_f64p = ct.POINTER(ct.c_double)

PFX_OK = 0
PFX_ERR_ARG = 1
PFX_ERR_STEPS = 2
PFX_ERR_CUDA = 3
PFX_ERR_NO_ENDPOINT = 4
PFX_ERR_TOO_LARGE = 5
PFX_ERR_NO_DEVICE = 6

PFX_FP64 = 0
PFX_FP32 = 1
PFX_BATCH_TILE_COST = 0x100
PFX_BATCH_COST_FMA = 0x200

NO_ENDPOINT_MSG = "Stage 2: No valid endpoint found on global top/right edges."

BUF = dict(EDGE_D=0, EDGE_P=1, BACKPTR=2, EDGE_CF=3, VALID=4, D_ARR=5, L_ARR=6,
           TOP_D=7, TOP_L=8, RIGHT_D=9, RIGHT_L=10, SEG_NORM=11, SEG_META=12,
           D_PROP=13, L_PROP=14, COST=15, FEAT_BF16=16)

# (name, restype, argtypes) for every exported symbol of the header
SIGNATURES = [
    ("pfx_status_string", ct.c_char_p, [ct.c_int]),
    ("pfx_last_error", ct.c_char_p, []),
    ("pfx_version", ct.c_int, []),
    ("pfx_kernel_launches", ct.c_int64, []),
    ("pfx_plan_create", ct.c_int, [_i64, _i64, _i32, _i64p, _f64p, _i32, ct.POINTER(_vp)]),
    ("pfx_plan_create_ex", ct.c_int, [_i64, _i64, _i32, _i64p, _f64p, _i32, _i32,
                                      ct.POINTER(_vp)]),
    ("pfx_plan_destroy", None, [_vp]),
    ("pfx_plan_info", ct.c_int, [_vp, _i64p]),
    ("pfx_plan_set_warps", ct.c_int, [_vp, _i32]),
    ("pfx_plan_buffer", ct.c_int, [_vp, ct.c_int, ct.POINTER(_vp), _i64p]),
    ("pfx_plan_load_cost", ct.c_int, [_vp, _vp, _i64, _vp]),
    ("pfx_plan_load_features", ct.c_int, [_vp, _vp, _vp, _i32, _vp]),
    ("pfx_plan_load_cost_f32", ct.c_int, [_vp, _vp, _i64, _vp]),
    ("pfx_plan_load_features_bf16", ct.c_int, [_vp, _vp, _vp, _i32, _vp]),
    ("pfx_plan_set_tile_mask", ct.c_int, [_vp, _vp, _i32, _vp]),
    ("pfx_plan_set_tile_range", ct.c_int, [_vp, _i32, _i32, _vp]),
    ("pfx_stage1", ct.c_int, [_vp, _vp, _i64, _vp]),
    ("pfx_stage2_propagate", ct.c_int, [_vp, _vp, _i64, _vp]),
    ("pfx_stage2_edges", ct.c_int, [_vp, _vp, _i64, _vp]),
    ("pfx_stage2_prop", ct.c_int, [_vp, _vp]),
    ("pfx_snapshot_prop", ct.c_int, [_vp, _vp]),
    ("pfx_stage2_scan", ct.c_int, [_vp, _f64, _vp]),
    ("pfx_stage2_stitch", ct.c_int, [_vp, ct.c_int, _i64, _i64, _i64, _i64, _vp]),
    ("pfx_stage2_chain", ct.c_int, [_vp, ct.c_int, _i64, _i64, _i64, _i64, _i32p, _i32,
                                    _i32p, _vp]),
    ("pfx_parflex_device", ct.c_int, [_vp, _vp, _i64, _f64, _vp]),
    ("pfx_result", ct.c_int, [_vp, _vp, _f64p, _i64p, _i64p]),
    ("pfx_copy_path", ct.c_int, [_vp, _vp, _i64p, _i64]),
    ("pfx_parflex", ct.c_int, [_f64p, _i64, _i64, _i64, _i64p, _f64p, _i32, _f64,
                               _i32, _f64p, _i64p, _i64, _i64p]),
    ("pfx_cost_matrix_f64", ct.c_int, [_vp, _vp, _i32, _i64, _i64, _vp, _vp, _i64, _vp]),
    ("pfx_flexdtw_tile", ct.c_int, [_vp, _i64, _i32, _i32, _i64p, _f64p, _i32, _vp, _vp,
                                    _vp, _vp]),
    ("pfx_flexdtw_tile_noalloc", ct.c_int, [_vp, _i64, _i32, _i32, _i64p, _f64p, _i32, _vp,
                                            _vp, _vp, _vp]),
    ("pfx_batch_create", ct.c_int, [_i32, _i64p, _i64p, _i32p, _i64p, _f64p, _i32, _i32, _i64,
                                    _i32, _i32, ct.POINTER(_vp)]),
    ("pfx_batch_destroy", None, [_vp]),
    ("pfx_batch_info", ct.c_int, [_vp, _i64p]),
    ("pfx_batch_features", ct.c_int, [_vp, _i32, ct.POINTER(_vp), ct.POINTER(_vp)]),
    ("pfx_batch_load_async", ct.c_int, [_vp, _i32, _vp, _vp, _vp]),
    ("pfx_batch_plan", ct.c_int, [_vp, _i32, ct.POINTER(_vp)]),
    ("pfx_batch_set_masks", ct.c_int, [_vp, _vp, _i32, _vp]),
    ("pfx_batch_complete", ct.c_int, [_vp, _i32, _f64, _vp, _vp]),
    ("pfx_batch_run", ct.c_int, [_vp, _f64, _i32, _vp]),
    ("pfx_batch_timing", ct.c_int, [_vp, _f64p]),
    ("pfx_batch_results", ct.c_int, [_vp, _vp, _f64p, _i64p, _i64p]),
    ("pfx_batch_copy_paths", ct.c_int, [_vp, _vp, _i64p, _i64p, _i64]),
    ("pfx_batch_copy_paths_rows", ct.c_int, [_vp, _vp, _i64p, _i64p, _i64p, _i64]),
    ("pfx_batch_check_paths", ct.c_int, [_vp, _i32, _vp, _vp, _vp]),
    ("pfx_pool_features", ct.c_int, [_vp, _i32, _i64, _i32, _vp, _vp]),
    ("pfx_pooled_cost", ct.c_int, [_vp, _vp, _i32, _i64, _i64, _vp, _vp]),
    ("pfx_pooled_center", ct.c_int, [_vp, _i64, _i64, _vp, _vp]),
    ("pfx_pooled_center_features", ct.c_int, [_vp, _vp, _i32, _i64, _i64, _vp, _vp]),
    ("pfx_pooled_center_scratch", ct.c_int64, [_i64, _i64]),
    ("pfx_conv3x3_forward_features", ct.c_int, [_vp, _vp, _i32, _i32, _i32, _vp, _vp, _i32,
                                                _i32, _i32, _vp, _i32, _vp]),
    ("pfx_conv3x3_forward", ct.c_int, [_vp, _i32, _i32, _i32, _i32, _vp, _vp, _i32, _i32, _i32,
                                       _vp, _i32, _vp]),
    ("pfx_conv3x3_backward", ct.c_int, [_vp, _i32, _i32, _i32, _vp, _i32, _i32, _vp, _i32, _vp,
                                        _vp, _vp, _vp, _vp]),
    ("pfx_tile_max", ct.c_int, [_vp, _i32, _i32, _i32, _i32, _i64, _i64, _i64, _i64, _i32, _vp,
                                _vp, _vp]),
    ("pfx_tile_bce", ct.c_int, [_vp, _vp, _i32, ct.c_float, _vp, _vp, _vp]),
    ("pfx_tile_max_backward", ct.c_int, [_vp, _vp, _i32, _vp, _vp]),
    ("pfx_adam_step", ct.c_int, [_vp, _vp, _vp, _vp, _i64, ct.c_float, ct.c_float, ct.c_float,
                                 ct.c_float, _i32, _vp]),
    ("pfx_tile_mask_from_scores", ct.c_int, [_vp, _i32, _i32, ct.c_float, _i32, _i32, _vp,
                                             _vp]),
]

_lib = None
_lock = threading.Lock()


class PfxError(RuntimeError):
    """A device-side failure reported by the library (CUDA error)."""


def load(build_if_missing: bool = False):
    """Load the shared library (optionally building it first)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.LIB_PATH
        if not os.path.exists(path):
            if build_if_missing:
                _build.build()
            else:
                raise RuntimeError(
                    f"parflexdtw_b200 CUDA library not built ({path}); run "
                    "`python -m parflexdtw_b200.build` (there is no CPU fallback)")
        lib = ct.CDLL(path)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(status: int):
    """Map a pfx_status to the reference's exception types."""
    if status == PFX_OK:
        return
    lib = load()
    msg = lib.pfx_last_error().decode(errors="replace")
    if status == PFX_ERR_NO_ENDPOINT:
        raise ValueError(NO_ENDPOINT_MSG)
    if status in (PFX_ERR_ARG, PFX_ERR_STEPS, PFX_ERR_TOO_LARGE):
        raise ValueError(msg)
    if status == PFX_ERR_NO_DEVICE:
        raise RuntimeError("parflexdtw_b200 needs a CUDA device: " + msg)
    raise PfxError(msg)


def i64_array(values):
    arr = (ct.c_int64 * len(values))(*[int(v) for v in values])
    return arr


def i32_array(values):
    return (ct.c_int32 * len(values))(*[int(v) for v in values])


def f64_array(values):
    return (ct.c_double * len(values))(*[float(v) for v in values])
