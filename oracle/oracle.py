"""ctypes wrapper around the C restatement in ``parflex_oracle.c``.

TEST INFRASTRUCTURE ONLY: the oracle the device path is checked against and
the CPU baseline bench.py times beside it.  Only tests/, the smoke check in
``__graft_entry__`` and bench.py's CPU-baseline leg import this module.

Build with ``python oracle/build_oracle.py`` (or ``__graft_entry__.build()``);
the library lands in ``oracle/_build/liboracle.so``.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_f64p = ct.POINTER(ct.c_double)
_f32p = ct.POINTER(ct.c_float)
_i64p = ct.POINTER(ct.c_int64)
_i32p = ct.POINTER(ct.c_int32)
_u8p = ct.POINTER(ct.c_uint8)
_i8p = ct.POINTER(ct.c_int8)


class _Result(ct.Structure):
    _fields_ = [
        ("N", ct.c_int64), ("M", ct.c_int64), ("L", ct.c_int64),
        ("hop", ct.c_int64), ("n1", ct.c_int64), ("n2", ct.c_int64),
        ("edge_Df", _f64p), ("edge_S", _i32p),
        ("edge_start_r", _i64p), ("edge_start_c", _i64p),
        ("edge_Cf_olap", _f64p), ("edge_lens", _i64p),
        ("valid_mask", _u8p), ("tile_B", ct.POINTER(_i8p)),
        ("tile_best", _f64p), ("tile_wp_len", _i64p),
        ("D_prop", _f64p), ("L_prop", _f64p),
        ("D_arr", _f64p), ("L_arr", _f64p),
        ("top_D", _f64p), ("top_L", _f64p),
        ("right_D", _f64p), ("right_L", _f64p),
        ("max_segs", ct.c_int64),
        ("seg_best_norm", _f64p), ("seg_best_meta", _i64p),
        ("best_cost", ct.c_double), ("best_end", ct.c_int64 * 6),
        ("found", ct.c_int64),
        ("wp", _i64p), ("wp_len", ct.c_int64),
        ("tile_order", _i64p), ("n_stitch", ct.c_int64),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library not built: {LIB_PATH} "
                               "(run python oracle/build_oracle.py)")
        L = ct.CDLL(LIB_PATH)
        L.oracle_parflex.restype = ct.c_int
        L.oracle_parflex.argtypes = [_f64p, ct.c_int64, ct.c_int64, ct.c_int64,
                                     _i64p, _f64p, ct.c_int, ct.c_double,
                                     ct.c_int64, ct.c_int, ct.c_int,
                                     ct.POINTER(_Result)]
        L.oracle_parflex2.restype = ct.c_int
        L.oracle_parflex2.argtypes = [_f64p, ct.c_int64, ct.c_int64, ct.c_int64,
                                      _i64p, _f64p, ct.c_int, ct.c_double,
                                      ct.c_int64, ct.c_int, ct.c_int, ct.c_int,
                                      ct.POINTER(_Result)]
        L.oracle_tile_dp_f32.argtypes = [_f32p, ct.c_int64, ct.c_int64, ct.c_int64,
                                         _i64p, _f64p, ct.c_int, _f32p, _i32p, _i8p]
        L.oracle_free.argtypes = [ct.POINTER(_Result)]
        L.oracle_result_size.restype = ct.c_int64
        L.oracle_tile_dp.argtypes = [_f64p, ct.c_int64, ct.c_int64, ct.c_int64,
                                     _i64p, _f64p, ct.c_int, _f64p, _i32p, _i8p]
        L.oracle_find_best_endpoint.restype = ct.c_double
        L.oracle_find_best_endpoint.argtypes = [_f64p, _i32p, ct.c_int64,
                                                ct.c_int64, ct.c_int64, _i64p,
                                                _i64p]
        L.oracle_backtrace_tile.restype = ct.c_int64
        L.oracle_backtrace_tile.argtypes = [_i8p, ct.c_int64, ct.c_int64, _i64p,
                                            ct.c_int, ct.c_int64, ct.c_int64,
                                            _i64p]
        L.oracle_cost_fma.argtypes = [_f64p, _f64p, ct.c_int, ct.c_int64, ct.c_int64, _f64p]
        if L.oracle_result_size() != ct.sizeof(_Result):
            raise RuntimeError("oracle_result layout mismatch")
        _lib = L
    return _lib


def _ptr(a, t):
    return a.ctypes.data_as(t)


def cost_matrix_fma(F1, F2):
    """The device's FMA cost mode on the host: L2-normalised features
    (``workloads.l2norm``), then C = 1 - sum_f a_f b_f as a fixed-order chain
    of fused multiply-adds (``oracle_cost_fma``)."""
    from parflexdtw_b200.workloads import l2norm
    A = np.ascontiguousarray(l2norm(np.asarray(F1, dtype=np.float64)))
    B = np.ascontiguousarray(l2norm(np.asarray(F2, dtype=np.float64)))
    d, N = A.shape
    M = B.shape[1]
    C = np.empty((N, M), dtype=np.float64)
    lib().oracle_cost_fma(_ptr(A, _f64p), _ptr(B, _f64p), d, N, M, _ptr(C, _f64p))
    return C


def _steps_weights(steps, weights):
    st = np.ascontiguousarray(np.asarray(steps, dtype=np.int64).reshape(-1, 2))
    w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).reshape(-1))
    if st.shape[0] != w.shape[0]:
        raise ValueError("steps and weights differ in length")
    return st, w


def flexdtw(C, steps, weights, buffer=1, fp32=False):
    """``FlexDTW.flexdtw`` restated: returns (best_cost, wp, D, P, B).

    ``fp32``: the FP32 form (C rounded to FP32, DP values in FP32; D is
    returned widened to FP64)."""
    C = np.ascontiguousarray(C, dtype=np.float64)
    R, W = C.shape
    st, w = _steps_weights(steps, weights)
    D = np.empty((R, W), np.float64)
    P = np.empty((R, W), np.int32)
    B = np.empty((R, W), np.int8)
    L = lib()
    if fp32:
        Cf = np.ascontiguousarray(C, dtype=np.float32)
        Df = np.empty((R, W), np.float32)
        L.oracle_tile_dp_f32(_ptr(Cf, _f32p), W, R, W, _ptr(st, _i64p), _ptr(w, _f64p),
                             st.shape[0], _ptr(Df, _f32p), _ptr(P, _i32p), _ptr(B, _i8p))
        D[...] = Df
    else:
        L.oracle_tile_dp(_ptr(C, _f64p), W, R, W, _ptr(st, _i64p), _ptr(w, _f64p),
                         st.shape[0], _ptr(D, _f64p), _ptr(P, _i32p), _ptr(B, _i8p))
    br, bc = ct.c_int64(), ct.c_int64()
    best = L.oracle_find_best_endpoint(_ptr(D, _f64p), _ptr(P, _i32p), R, W,
                                       int(buffer), ct.byref(br), ct.byref(bc))
    out = np.empty((R + W + 4, 2), np.int64)
    k = L.oracle_backtrace_tile(_ptr(B, _i8p), R, W, _ptr(st, _i64p),
                                st.shape[0], br.value, bc.value,
                                _ptr(out, _i64p))
    return best, out[:k].T.copy(), D, P, B


def _arr(p, n, dtype):
    if n == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(p, shape=(n,)).astype(dtype, copy=True)


def parflex_full(C, steps, weights, beta, L, threads=0, tile_wp=False, fp32=False):
    """Run the restated ParFlex and return every intermediate as numpy arrays.

    ``fp32``: the FP32 form -- C rounded to FP32 and the tile DP in FP32,
    stage 2 in FP64 on the widened values.  Raises ``ValueError`` with the
    reference's wording when no endpoint is found (``Parflex.py:1285-1286``).
    """
    C = np.ascontiguousarray(C, dtype=np.float64)
    if fp32:
        C = C.astype(np.float32).astype(np.float64)
    N, M = C.shape
    st, w = _steps_weights(steps, weights)
    res = _Result()
    lb = lib()
    rc = lb.oracle_parflex2(_ptr(C, _f64p), N, M, M, _ptr(st, _i64p),
                            _ptr(w, _f64p), st.shape[0], float(beta), int(L),
                            int(threads), int(bool(tile_wp)), int(bool(fp32)),
                            ct.byref(res))
    try:
        if rc == -2:
            raise ValueError("Stage 2: No valid endpoint found on global "
                             "top/right edges.")
        if rc != 0:
            raise RuntimeError(f"oracle_parflex failed ({rc})")
        n1, n2, Lb = res.n1, res.n2, res.L
        n4 = n1 * n2 * 2 * Lb
        s4 = (n1, n2, 2, Lb)
        ms = res.max_segs
        out = dict(
            n1=n1, n2=n2, L=Lb,
            edge_Df=_arr(res.edge_Df, n4, np.float64).reshape(s4),
            edge_S=_arr(res.edge_S, n4, np.int32).reshape(s4),
            edge_start_r=_arr(res.edge_start_r, n4, np.int64).reshape(s4),
            edge_start_c=_arr(res.edge_start_c, n4, np.int64).reshape(s4),
            edge_Cf_olap=_arr(res.edge_Cf_olap, n4, np.float64).reshape(s4),
            edge_lens=_arr(res.edge_lens, n1 * n2 * 2, np.int64).reshape(n1, n2, 2),
            valid_mask=_arr(res.valid_mask, n4, np.uint8).reshape(s4).astype(bool),
            D_prop=_arr(res.D_prop, n4, np.float64).reshape(s4),
            L_prop=_arr(res.L_prop, n4, np.float64).reshape(s4),
            D_arr=_arr(res.D_arr, n4, np.float64).reshape(s4),
            L_arr=_arr(res.L_arr, n4, np.float64).reshape(s4),
            top_D=_arr(res.top_D, M, np.float64),
            top_L=_arr(res.top_L, M, np.float64),
            right_D=_arr(res.right_D, N, np.float64),
            right_L=_arr(res.right_L, N, np.float64),
            seg_best_norm=_arr(res.seg_best_norm, 2 * ms, np.float64).reshape(2, ms),
            seg_best_meta=_arr(res.seg_best_meta, 12 * ms, np.int64).reshape(2, ms, 6),
            best_cost=float(res.best_cost),
            best_end=tuple(int(x) for x in res.best_end),
            wp=_arr(res.wp, 2 * res.wp_len, np.int64).reshape(-1, 2).T.copy(),
            tile_order=_arr(res.tile_order, 4 * res.n_stitch, np.int64).reshape(-1, 4),
        )
        if tile_wp:
            out["tile_best"] = _arr(res.tile_best, n1 * n2, np.float64).reshape(n1, n2)
            out["tile_wp_len"] = _arr(res.tile_wp_len, n1 * n2, np.int64).reshape(n1, n2)
        return out
    finally:
        lb.oracle_free(ct.byref(res))


def parflex(C, steps, weights, beta, L, threads=0):
    """``Parflex.parflex`` restated: ``(best_cost, wp[2, K])``."""
    r = parflex_full(C, steps, weights, beta, L, threads=threads)
    wp = r["wp"]
    if wp.size == 0:
        wp = np.array([[], []], dtype=np.int64)
    return r["best_cost"], wp
