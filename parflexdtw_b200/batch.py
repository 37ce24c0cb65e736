"""Batched alignment: many pairs of uneven lengths through one device batch.

``parflex_batch(pairs, steps, weights, beta, L=None)`` aligns every pair and
returns, per pair, what ``parflex`` returns for it: ``(best_cost, wp[2, K])``.
The reference has no batch entry point -- its notebooks loop over pairs
calling ``tiled_stage1_from_features`` + ``run_stage2_from_tiled`` or
``parflex`` (Parflex.py:1466-1547, gpu_flexdtw.py:405-470) -- so the result
of each pair is, by construction, that of those calls.

Device side (``pfx_batch_*`` in include/parflexdtw_b200.h): one arena holds
every pair's plan.  Pairs are packed into waves whose cost slabs fit a
memory pool; per wave the cost of each pair is built from its features by
the cost kernels, then ONE persistent stage-1 launch runs all tiles of all
pairs of the wave from a device work queue.  With ``cost="tile"`` (FP64,
d <= 16) the stage-1 kernel builds each tile's cost itself, into one cost
slab per resident CTA, and ONE launch runs every tile of every pair
whatever the batch's size.  Stage 2 runs on forked streams.  The whole
launch sequence is recorded once into a CUDA graph and replayed.
"""
from __future__ import annotations

import ctypes as ct
import weakref

import numpy as np
import torch

from . import _lib
from .plan import Plan, _DevView, current_stream_ptr, normalize_steps

_I64P = ct.POINTER(ct.c_int64)


def _free_batch(handle):
    if handle:
        _lib.load().pfx_batch_destroy(handle)


class Batch:
    """Owner of a ``pfx_batch*``: shapes, tile lengths, steps and weights are
    fixed at creation; features are loaded and the batch re-run any number
    of times (the CUDA graph is recorded on the first run)."""

    def __init__(self, shapes, L_per_pair, steps, weights, d, wave_bytes=0, warps=0,
                 precision="fp64", cost="slabs", cost_fma=False):
        lib = _lib.load()
        if precision not in ("fp64", "fp32"):
            raise ValueError("precision must be 'fp64' or 'fp32'")
        if cost not in ("slabs", "tile"):
            raise ValueError("cost must be 'slabs' (separate cost kernels, in waves) or 'tile' "
                             "(FP64, d <= 16: built inside the stage-1 kernel, tile by tile)")
        if cost_fma and (precision != "fp64" or cost != "slabs"):
            raise ValueError("cost_fma needs precision='fp64' and cost='slabs'")
        # True: the FP64 cost as a fixed-order FMA chain (PFX_BATCH_COST_FMA)
        self.cost_fma = bool(cost_fma)
        self.precision = precision
        if not torch.cuda.is_available():
            raise RuntimeError("parflexdtw_b200 needs a CUDA device")
        torch.cuda.init()
        st, w = normalize_steps(steps, weights)
        self.steps, self.weights = st, w
        self.shapes = [(int(n), int(m)) for n, m in shapes]
        n = len(self.shapes)
        if n == 0:
            raise ValueError("empty batch")
        Ls = list(L_per_pair) if np.ndim(L_per_pair) else [int(L_per_pair)] * n
        if len(Ls) != n:
            raise ValueError("one tile length per pair")
        self.L = [int(x) for x in Ls]
        self.d = int(d)
        h = ct.c_void_p()
        _lib.check(lib.pfx_batch_create(
            n, _lib.i64_array([s[0] for s in self.shapes]), _lib.i64_array([s[1] for s in self.shapes]),
            _lib.i32_array(self.L), _lib.i64_array(st.reshape(-1)), _lib.f64_array(w), st.shape[0],
            self.d, int(wave_bytes), int(warps),
            (_lib.PFX_FP32 if precision == "fp32" else _lib.PFX_FP64) |
            (_lib.PFX_BATCH_TILE_COST if cost == "tile" else 0) |
            (_lib.PFX_BATCH_COST_FMA if cost_fma else 0), ct.byref(h)))
        self._h = h
        self._fin = weakref.finalize(self, _free_batch, h)
        info = (ct.c_int64 * 9)()
        _lib.check(lib.pfx_batch_info(h, info))
        (self.n, self.waves, self.tiles, self.cells, self.device_bytes, self.warps,
         self.max_wave_tiles, self.slab_bytes, gen) = (int(x) for x in info)
        # True: stage 1 builds each tile's cost itself (one wave, one slab per CTA)
        self.cost_in_kernel = bool(gen)
        self.device = torch.cuda.current_device()
        self._plans = {}

    @property
    def handle(self):
        return self._h

    def close(self):
        self._plans.clear()
        self._fin()

    def feature_views(self, i):
        """Device tensors (d x N_i, d x M_i) that pair i's features are read from."""
        p1, p2 = ct.c_void_p(), ct.c_void_p()
        _lib.check(_lib.load().pfx_batch_features(self._h, int(i), ct.byref(p1), ct.byref(p2)))
        N, M = self.shapes[i]
        dev = f"cuda:{self.device}"
        a = torch.as_tensor(_DevView(p1.value, (self.d, N), "<f8"), device=dev)
        b = torch.as_tensor(_DevView(p2.value, (self.d, M), "<f8"), device=dev)
        a._pfx_owner = self
        b._pfx_owner = self
        return a, b

    def load(self, pairs, non_blocking=True):
        """Copy every pair's features (host arrays or tensors, d x frames)
        into the batch's device buffers on the current stream."""
        if len(pairs) != self.n:
            raise ValueError(f"{len(pairs)} pairs for a batch of {self.n}")
        for i, (F1, F2) in enumerate(pairs):
            a, b = self.feature_views(i)
            for dst, src in ((a, F1), (b, F2)):
                t = src if isinstance(src, torch.Tensor) else torch.from_numpy(
                    np.ascontiguousarray(src, dtype=np.float64))
                if tuple(t.shape) != tuple(dst.shape):
                    raise ValueError(f"pair {i}: features {tuple(t.shape)} for a buffer "
                                     f"{tuple(dst.shape)}")
                dst.copy_(t, non_blocking=non_blocking)

    def set_masks(self, masks, stream=None):
        """Restrict each pair to its tile mask (a CUDA uint8 tensor holding
        the pairs' (n1, n2) masks concatenated in pair order)."""
        m = masks.to(torch.uint8).contiguous()
        _lib.check(_lib.load().pfx_batch_set_masks(self._h, ct.c_void_p(m.data_ptr()), 1,
                                                   stream or current_stream_ptr()))
        info = (ct.c_int64 * 9)()
        _lib.check(_lib.load().pfx_batch_info(self._h, info))
        self.waves = int(info[1])
        self.masked = True

    def complete(self, i, beta, tiles=None, stream=None):
        """After a masked run: pair i again with `tiles` ((n1, n2) bool,
        host) added to its run, or every tile (None: the full-tile method);
        stage 1 runs only on tiles that have not run.  Returns
        (best_cost, (K, 2) path)."""
        ptr = None
        if tiles is not None:
            tiles = np.ascontiguousarray(tiles, dtype=np.uint8).reshape(-1)
            ptr = tiles.ctypes.data
        _lib.check(_lib.load().pfx_batch_complete(self._h, int(i), float(beta), ptr,
                                                  stream or current_stream_ptr()))
        p = self.plan(i)
        best, end, found, n = p.result()
        return best, p.path(n)

    def run(self, beta, use_graph=True, stream=None):
        """Aligns every pair (asynchronous on the current stream)."""
        _lib.check(_lib.load().pfx_batch_run(self._h, float(beta), 1 if use_graph else 0,
                                       stream or current_stream_ptr()))

    def timing(self):
        """(cost_ms, stage1_ms, stage2_ms) of the last ``run(use_graph=False)``."""
        ms = (ct.c_double * 3)()
        _lib.check(_lib.load().pfx_batch_timing(self._h, ms))
        return tuple(float(x) for x in ms)

    def results(self, stream=None):
        """(best_cost[n], best_end[n, 7], wp_len[n]); synchronises."""
        best = np.zeros(self.n, dtype=np.float64)
        end = np.zeros((self.n, 7), dtype=np.int64)
        lens = np.zeros(self.n, dtype=np.int64)
        _lib.check(_lib.load().pfx_batch_results(
            self._h, stream or current_stream_ptr(),
            best.ctypes.data_as(ct.POINTER(ct.c_double)), end.ctypes.data_as(_I64P),
            lens.ctypes.data_as(_I64P)))
        return best, end, lens

    def paths(self, lens, stream=None):
        """Every pair's stitched path as (K_i, 2) int64 arrays, start first."""
        lens = np.asarray(lens, dtype=np.int64)
        offs = np.zeros(self.n, dtype=np.int64)
        if self.n > 1:
            offs[1:] = np.cumsum(lens)[:-1]
        total = max(int(lens.sum()), 1)
        # page-locked staging (kept between calls), then one copy per path
        if getattr(self, "_pinned", None) is None or self._pinned.shape[0] < total:
            self._pinned = torch.empty((int(total * 1.25) + 1024, 2), dtype=torch.int64,
                                       pin_memory=True)
        stage = self._pinned.numpy()
        _lib.check(_lib.load().pfx_batch_copy_paths(
            self._h, stream or current_stream_ptr(), stage.ctypes.data_as(_I64P),
            offs.ctypes.data_as(_I64P), stage.shape[0]))
        return [stage[o:o + k].copy() for o, k in zip(offs, lens)]

    def paths_rows(self, lens, stream=None):
        """Every pair's stitched path as a (2, K_i) int64 array (rows, then
        columns; the reference's ``wp`` layout), from one device gather and
        one copy into a fresh host array (the arrays are views of it)."""
        lens = np.asarray(lens, dtype=np.int64)
        offs = np.zeros(self.n, dtype=np.int64)
        if self.n > 1:
            offs[1:] = np.cumsum(lens)[:-1]
        total = int(lens.sum())
        # page-locked (torch's caching host allocator reuses the block once
        # the arrays are dropped), so the copy runs at full link speed
        flat = torch.empty(max(2 * total, 2), dtype=torch.int64, pin_memory=True).numpy()
        _lib.check(_lib.load().pfx_batch_copy_paths_rows(
            self._h, stream or current_stream_ptr(), flat.ctypes.data_as(_I64P),
            offs.ctypes.data_as(_I64P), lens.ctypes.data_as(_I64P), max(total, 1)))
        return [flat[2 * o:2 * o + 2 * k].reshape(2, k) for o, k in zip(offs, lens)]

    def check_paths(self, margin, stream=None):
        """Masked batch, after a run: (near, flags) on the device -- per tile
        (pairs' (n1, n2) arrays concatenated) 1 where a tile not run lies
        within about `margin` cells of the pair's path, per pair 1 where any
        does (``pfx_batch_check_paths``)."""
        near = torch.empty(self.tiles, dtype=torch.uint8, device=f"cuda:{self.device}")
        flags = torch.empty(self.n, dtype=torch.int32, device=f"cuda:{self.device}")
        _lib.check(_lib.load().pfx_batch_check_paths(
            self._h, int(margin), ct.c_void_p(near.data_ptr()), ct.c_void_p(flags.data_ptr()),
            stream or current_stream_ptr()))
        return near, flags

    def plan(self, i) -> Plan:
        """Pair i's plan (borrowed from the batch: stage-2 buffers, results)."""
        if i not in self._plans:
            h = ct.c_void_p()
            _lib.check(_lib.load().pfx_batch_plan(self._h, int(i), ct.byref(h)))
            N, M = self.shapes[i]
            self._plans[i] = Plan.borrow(h, self, N, M, self.L[i], self.steps, self.weights)
        return self._plans[i]


def _split_pair(pair):
    if isinstance(pair, (tuple, list)) and len(pair) == 2:
        return pair
    raise ValueError("parflex_batch takes (F1, F2) feature pairs (d x frames each)")


def parflex_batch(pairs, steps, weights, beta, L=None, wave_bytes=0, warps=0,
                  use_graph=True, errors="raise", tuner=None, precision="fp64", cost="slabs",
                  cost_fma=False):
    """ParFlex on every (F1, F2) feature pair of ``pairs`` in one device batch.

    Same argument conventions as ``parflex`` (features are d x frames, the
    cost is 1 - L2norm(F1)^T L2norm(F2) as in tiled_stage1_from_features).
    ``L``: one tile length for all pairs, one per pair, or None to let the
    autotuner pick per length bucket.  ``precision="fp32"`` runs the FP32
    form (bf16 tensor-core cost, FP32 DP; d <= 256).  ``cost="tile"`` builds
    the FP64 cost inside the stage-1 kernel, tile by tile, in one launch
    instead of with separate cost kernels in waves (same results).
    ``cost_fma=True`` forms the FP64 cost as a fixed-order FMA chain (13 FP64
    operations per cell instead of 24; another deterministic rounding of the
    same cost).  Returns a list with, per pair,
    ``(best_cost, wp[2, K])``.  A pair whose scan finds no endpoint raises the
    reference's ValueError (``errors="raise"``) or yields None
    (``errors="none"``).
    """
    if errors not in ("raise", "none"):
        raise ValueError("errors must be 'raise' or 'none'")
    feats = [_split_pair(p) for p in pairs]
    if not feats:
        return []
    d = int(np.shape(feats[0][0])[0])
    shapes = []
    for F1, F2 in feats:
        if np.shape(F1)[0] != d or np.shape(F2)[0] != d:
            raise ValueError("all features must share the feature dimension")
        shapes.append((int(np.shape(F1)[1]), int(np.shape(F2)[1])))
    if L is None:
        from .autotune import default_tuner
        t = tuner or default_tuner()
        Ls, w = t.choose(shapes, steps, weights, d, precision=precision)
        warps = warps or w
    else:
        Ls = L
    b = Batch(shapes, Ls, steps, weights, d, wave_bytes=wave_bytes, warps=warps,
              precision=precision, cost=cost, cost_fma=cost_fma)
    b.load(feats)
    b.run(beta, use_graph=use_graph)
    best, end, lens = b.results()
    paths = b.paths(lens)
    out = []
    for i in range(b.n):
        if not end[i, 6]:
            if errors == "raise":
                raise ValueError(L_NO_ENDPOINT)
            out.append(None)
            continue
        wp = paths[i]
        out.append((float(best[i]), np.ascontiguousarray(wp.T) if wp.shape[0] else
                    np.array([[], []], dtype=np.int64)))
    b.close()
    return out


L_NO_ENDPOINT = _lib.NO_ENDPOINT_MSG
