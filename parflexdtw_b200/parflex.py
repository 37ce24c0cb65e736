"""Reference-compatible ParFlex API on the B200 device path.

Mirrors the public functions of the reference's ``Parflex_gpu.py`` /
``Parflex.py`` (same names, arguments, defaults, return shapes and error
messages):

* ``parflex(C, steps, weights, beta, L=None, ...) -> (best_cost, wp[2, K])``
  (Parflex_gpu.py:656-854, Parflex.py:1510-1547)
* ``tiled_stage1_from_features(F1, F2, steps=None, weights=None, beta=0.1,
  L=None, use_gpu=None) -> (C or None, tiled_result)`` (Parflex_gpu.py:610-653)
* ``run_stage2_from_tiled(tiled_result, C=None, beta=0.1, ...) -> dict``
  (Parflex_gpu.py:857-910)
* ``run_flexdtw_on_tiles(C, L, ...) -> (chunks_dict, L, n1, n2)``
  (Parflex_gpu.py:342-607)
* ``flexdtw_chunk_from_global_C(C_dev, L2_global, r0, r1, c0, c1, steps,
  weights, buffer=1.0) -> (best_cost, wp, D, P, B, debug)`` (gpu_flexdtw.py:288-402,
  returning the six values its callers unpack)

Everything runs on the GPU; there is no CPU path.  ``use_gpu=False`` (or the
``PARFLEX_DISABLE_GPU`` environment variable with ``use_gpu=None``) raises,
because this package has nothing to fall back to.  Per-tile full matrices
(``chunks_dict[(i, j)]['D']`` etc.) are materialised lazily, on first access,
by re-running that tile's DP with full outputs; stage 2 itself only uses the
tile edges and the packed backpointers, which never leave the device.
"""
from __future__ import annotations

import csv
import math
import os
import threading
import time
import warnings
from collections.abc import Mapping

import numpy as np
import torch

from . import _lib as L
from .plan import Plan, current_stream_ptr, normalize_steps

DEFAULT_CHUNK_LENGTH = 4000  # Parflex.py:126

_STD_STEPS = np.array([[1, 1], [1, 2], [2, 1]])


def is_gpu_available() -> bool:
    """True when a CUDA device is visible and the library loads."""
    try:
        L.load()
        return torch.cuda.is_available()
    except Exception:
        return False


def _require_gpu(use_gpu):
    if use_gpu is None:
        use_gpu = os.environ.get("PARFLEX_DISABLE_GPU", "").strip() == ""
    if not use_gpu:
        raise ValueError("parflexdtw_b200 has no CPU path (use_gpu=False or "
                         "PARFLEX_DISABLE_GPU set); use the reference package "
                         "for CPU runs")
    if not torch.cuda.is_available():
        raise RuntimeError("parflexdtw_b200 needs a CUDA device")
    L.load()


_STAGE_ELEMS = 1 << 25  # FP64 elements per pinned staging chunk (256 MB)
_STAGE_THREADS = 8      # host threads filling a chunk
# the two chunks, the filling threads, and per chunk the event after the last
# transfer out of it (kept across calls: a chunk is refilled only after it)
_stage = {"bufs": None, "pool": None, "done": [None, None]}
_stage_lock = threading.Lock()


def _upload_staged(arr: np.ndarray) -> torch.Tensor:
    """A large C-contiguous FP64 host array to the device through two reused
    page-locked chunks: while one chunk's copy to the device runs, host
    threads fill the other (numpy releases the GIL while copying), so the
    host copy and the transfer overlap."""
    from concurrent.futures import ThreadPoolExecutor
    if _stage["bufs"] is None:
        _stage["bufs"] = [torch.empty(_STAGE_ELEMS, dtype=torch.float64).pin_memory()
                          for _ in range(2)]
        _stage["pool"] = ThreadPoolExecutor(max_workers=_STAGE_THREADS)
    bufs, pool, done = _stage["bufs"], _stage["pool"], _stage["done"]
    out = torch.empty(arr.shape, dtype=torch.float64, device="cuda")
    src, dst = arr.reshape(-1), out.view(-1)
    n = src.size
    stream = torch.cuda.current_stream()
    for k, off in enumerate(range(0, n, _STAGE_ELEMS)):
        m = min(_STAGE_ELEMS, n - off)
        buf = bufs[k & 1]
        if done[k & 1] is not None:
            done[k & 1].synchronize()  # its previous transfer has read the chunk
        host = buf.numpy()
        part = -(-m // _STAGE_THREADS)
        futs = [pool.submit(np.copyto, host[a:min(a + part, m)],
                            src[off + a:off + min(a + part, m)])
                for a in range(0, m, part)]
        for f in futs:
            f.result()
        dst[off:off + m].copy_(buf[:m], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(stream)
        done[k & 1] = ev
    return out


def cost_matrix_to_gpu(C) -> torch.Tensor:
    """Host (or device) cost matrix as a contiguous FP64 CUDA tensor.  Host
    arrays above one staging chunk go through the double-buffered staged
    upload; smaller ones through one page-locked copy."""
    if isinstance(C, torch.Tensor):
        t = C if C.is_cuda else C.cuda()
        return t.to(torch.float64).contiguous()
    arr = np.ascontiguousarray(C, dtype=np.float64)
    if arr.size > _STAGE_ELEMS and arr.ndim == 2:
        with _stage_lock:
            return _upload_staged(arr)
    return torch.from_numpy(arr).pin_memory().cuda(non_blocking=True)


# the reference's name for the same upload (gpu_flexdtw.py:112-116); FP64 here
cost_matrix_to_gpu_f32 = cost_matrix_to_gpu


def cost_matrix_from_features_gpu(F1, F2) -> torch.Tensor:
    """``1 - L2norm(F1).T @ L2norm(F2)`` on the device in FP64, summed over
    the feature dimension in a fixed order (bit-identical on every run).
    ``F1`` is (d, N) and ``F2`` (d, M) (gpu_flexdtw.py:95-109)."""
    f1 = (F1 if isinstance(F1, torch.Tensor) else torch.from_numpy(
        np.ascontiguousarray(F1, dtype=np.float64))).cuda().to(torch.float64).contiguous()
    f2 = (F2 if isinstance(F2, torch.Tensor) else torch.from_numpy(
        np.ascontiguousarray(F2, dtype=np.float64))).cuda().to(torch.float64).contiguous()
    if f1.dim() != 2 or f2.dim() != 2 or f1.shape[0] != f2.shape[0]:
        raise ValueError("features must be (d, frames) with the same d")
    d, N = f1.shape
    M = f2.shape[1]
    C = torch.empty((N, M), dtype=torch.float64, device=f1.device)
    scratch = torch.empty(d * (N + M), dtype=torch.float64, device=f1.device)
    L.check(L.load().pfx_cost_matrix_f64(
        f1.data_ptr(), f2.data_ptr(), int(d), int(N), int(M), scratch.data_ptr(),
        C.data_ptr(), int(M), current_stream_ptr()))
    return C


def _features_to_device(F):
    t = F if isinstance(F, torch.Tensor) else torch.from_numpy(
        np.ascontiguousarray(F, dtype=np.float64))
    return t.cuda(non_blocking=True).to(torch.float64).contiguous()


class _CostSource:
    """The row-major FP64 cost matrix on the device: given, or computed from
    device features on first use (the plan itself holds the tile-skewed copy
    it works on, so the row-major matrix is only built when a caller asks for
    ``tiled_result['C_dev']`` or a per-tile ``chunks_dict`` record)."""

    def __init__(self, C_dev=None, F1=None, F2=None):
        self._C, self._F1, self._F2 = C_dev, F1, F2

    def get(self) -> torch.Tensor:
        if self._C is None:
            self._C = cost_matrix_from_features_gpu(self._F1, self._F2)
        return self._C


class TiledResult(dict):
    """``tiled_result`` dict; ``'C_dev'`` materialises on first access."""

    def __getitem__(self, k):
        v = dict.__getitem__(self, k)
        return v.get() if isinstance(v, _CostSource) else v

    def get(self, k, default=None):
        return self[k] if k in self else default


# ---------------------------------------------------------------------------
# per-tile helpers (FlexDTW.py:104-186 on a materialised tile)
# ---------------------------------------------------------------------------
def _find_best_endpoint(D, P, buffer):
    """find_best_endpoint (FlexDTW.py:104-154) on host arrays."""
    R, W = D.shape
    buf = int(buffer)
    rows = np.concatenate([np.full(W - buf, R - 1), np.arange(R - 2, buf - 1, -1)])
    cols = np.concatenate([np.arange(buf, W), np.full(max(R - 1 - buf, 0), W - 1)])
    p = P[rows, cols].astype(np.int64)
    rstart = np.where(p >= 0, 0, -p)
    cstart = np.where(p >= 0, p, 0)
    with np.errstate(divide="ignore", invalid="ignore"):
        avg = D[rows, cols] / ((rows - rstart) + (cols - cstart))
    best, br, bc = np.inf, -1, -1
    debug = []
    for k in range(rows.shape[0]):
        r, c, a = int(rows[k]), int(cols[k]), float(avg[k])
        if a < best:
            best, br, bc = a, r, c
        debug.append((c - W + 1, a, r, c) if r == R - 1 else (R - 1 - r, a, r, c))
    return best, br, bc, debug


def _backtrace_tile(B, steps, r, c):
    """backtrace_flexdtw (FlexDTW.py:161-186), start-first (2, K)."""
    path = [(r, c)]
    S = steps.shape[0]
    while r != 0 and c != 0:
        s = int(B[r, c])
        s = s + S if s < 0 else s
        r, c = r - int(steps[s, 0]), c - int(steps[s, 1])
        path.append((r, c))
    path.reverse()
    return np.array(path, dtype=np.int64).T


def _tile_full(C_dev: torch.Tensor, r0, r1, c0, c1, steps, weights):
    R, W = int(r1 - r0), int(c1 - c0)
    if R <= 0 or W <= 0:
        raise ValueError(f"Empty chunk: R={R}, C={W}")
    st, w = normalize_steps(steps, weights)
    dev = C_dev.device
    D = torch.empty((R, W), dtype=torch.float64, device=dev)
    P = torch.empty((R, W), dtype=torch.int32, device=dev)
    B = torch.empty((R, W), dtype=torch.int8, device=dev)
    base = C_dev.data_ptr() + (int(r0) * C_dev.stride(0) + int(c0)) * 8
    L.check(L.load().pfx_flexdtw_tile(
        base, C_dev.stride(0), R, W, L.i64_array(st.reshape(-1)), L.f64_array(w),
        st.shape[0], D.data_ptr(), P.data_ptr(), B.data_ptr(), current_stream_ptr()))
    return D.cpu().numpy(), P.cpu().numpy(), B.cpu().numpy()


def flexdtw_chunk_from_global_C(C_dev, L2_global, r0, r1, c0, c1, steps, weights,
                                buffer=1.0):
    """FlexDTW on ``C_dev[r0:r1, c0:c1]`` on the GPU (gpu_flexdtw.py:288-402).

    Returns ``(best_cost, wp, D, P, B, debug)`` -- the six values the
    reference's callers unpack -- as NumPy arrays matching
    ``FlexDTW.flexdtw`` (FP64, bit-exact).
    """
    C_dev = cost_matrix_to_gpu(C_dev)
    if int(L2_global) != C_dev.shape[1]:
        raise ValueError("L2_global must equal C_dev.shape[1]")
    D, P, B = _tile_full(C_dev, r0, r1, c0, c1, steps, weights)
    st, _ = normalize_steps(steps, weights)
    best, br, bc, debug = _find_best_endpoint(D, P, buffer)
    wp = _backtrace_tile(B, st, br, bc) if br >= 0 else np.zeros((2, 0), np.int64)
    return best, wp, D, P, B, debug


def flexdtw(C, steps, weights, buffer=1):
    """``FlexDTW.flexdtw`` (FlexDTW.py:326-378) on the GPU: the untiled
    FlexDTW of the whole cost matrix -- the accuracy baseline ParFlex
    approximates (with ``buffer = buffer_global(L1, L2, beta)``).  Returns
    ``(best_cost, wp[2, K], D, P, B, debug)`` as the reference does, bit-exact
    in FP64.  The DP runs as one device tile; D, P and B (13 bytes per cell)
    come back to the host for the endpoint search and the backtrace."""
    C_dev = cost_matrix_to_gpu(C)
    N, M = int(C_dev.shape[0]), int(C_dev.shape[1])
    return flexdtw_chunk_from_global_C(C_dev, M, 0, N, 0, M, steps, weights, buffer)


# ---------------------------------------------------------------------------
# lazy chunks_dict (Parflex.py:446-454 keys)
# ---------------------------------------------------------------------------
class _Chunk(Mapping):
    """One tile's record.  Geometry keys are eager; D / S / B / C / wp /
    best_cost / debug are computed on first access; the edge start sets come
    from the device edge tensors."""

    _KEYS = ("C", "D", "S", "B", "debug", "best_cost", "wp", "bounds", "hop",
             "shape", "starts_bot_edge", "starts_left_edge")

    def __init__(self, owner, i, j):
        import weakref
        self._o = weakref.proxy(owner)  # no reference cycle: the plan lease ends with owner
        self._i, self._j = i, j
        g = owner.plan
        s1, s2 = i * g.hop, j * g.hop
        e1, e2 = min(s1 + g.L, g.N), min(s2 + g.L, g.M)
        self._eager = {
            "bounds": (s1, e1, s2, e2),
            "hop": (g.hop if e1 < g.N else g.N - s1, g.hop if e2 < g.M else g.M - s2),
            "shape": (e1 - s1, e2 - s2),
        }
        self._lazy = {}

    def __getitem__(self, k):
        if k in self._eager:
            return self._eager[k]
        if k not in self._KEYS:
            raise KeyError(k)
        if k not in self._lazy:
            self._materialise(k)
        return self._lazy[k]

    def __iter__(self):
        return iter(self._KEYS)

    def __len__(self):
        return len(self._KEYS)

    def _materialise(self, k):
        o = self._o
        s1, e1, s2, e2 = self._eager["bounds"]
        if k in ("starts_bot_edge", "starts_left_edge"):
            bot, left = o.edge_start_sets(self._i, self._j)
            self._lazy["starts_bot_edge"] = bot
            self._lazy["starts_left_edge"] = left
        elif k == "C":
            self._lazy["C"] = o.C_dev[s1:e1, s2:e2].cpu().numpy()
        else:
            D, P, B = _tile_full(o.C_dev, s1, e1, s2, e2, o.plan.steps, o.plan.weights)
            best, br, bc, debug = _find_best_endpoint(D, P, 1)
            wp = (_backtrace_tile(B, o.plan.steps, br, bc) if br >= 0
                  else np.zeros((2, 0), np.int64))
            self._lazy.update(D=D, S=P, B=B, best_cost=best, wp=wp, debug=debug)


class ChunksDict(Mapping):
    """``chunks_dict`` keyed by ``(i, j)`` over a device stage-1 result."""

    def __init__(self, plan: Plan, cost):
        self.plan = plan
        self._cost = cost if isinstance(cost, _CostSource) else _CostSource(C_dev=cost)
        self._edgeP = None
        self._chunks = {(i, j): _Chunk(self, i, j)
                        for i in range(plan.n1) for j in range(plan.n2)}

    @property
    def C_dev(self) -> torch.Tensor:
        return self._cost.get()

    def __getitem__(self, k):
        return self._chunks[k]

    def __iter__(self):
        return iter(self._chunks)

    def __len__(self):
        return len(self._chunks)

    def edge_start_sets(self, i, j):
        """_edge_starts_from_S (Parflex.py:347-373) from the edge tensors."""
        if self._edgeP is None:
            self._edgeP = self.plan.host("EDGE_P")
        R, W = self._chunks[(i, j)]["shape"]
        vals = np.concatenate([self._edgeP[i, j, 0, :W], self._edgeP[i, j, 1, :R]])
        bot = {int(v) for v in vals if v > 0}
        left = {abs(int(v)) for v in vals if v <= 0}
        return bot, left


class _LazyList(list):
    pass


def _blocks(chunks: ChunksDict):
    """``tiled_result['blocks']`` (Parflex.py:1376-1395).  A FlexDTW tile with
    finite costs always has a non-empty path, so every tile is a block;
    ``S_single`` materialises on access."""
    out = _LazyList()
    for (i, j), ch in chunks.items():
        s1, e1, s2, e2 = ch["bounds"]
        out.append(_Block(ch, {"bi": i, "bj": j, "rows": (int(s1), int(e1)),
                               "cols": (int(s2), int(e2)), "Ck_shape": ch["shape"]}))
    return out


class _Block(Mapping):
    def __init__(self, chunk, eager):
        self._c = chunk
        self._e = eager

    def __getitem__(self, k):
        if k == "S_single":
            return self._c["S"]
        return self._e[k]

    def __iter__(self):
        return iter(list(self._e) + ["S_single"])

    def __len__(self):
        return len(self._e) + 1


# ---------------------------------------------------------------------------
# profiling CSVs (same file names and columns as the reference)
# ---------------------------------------------------------------------------
class _Phases:
    def __init__(self, enabled):
        self.enabled = enabled
        self.rows = []
        self._ev = []

    def mark(self, name):
        if not self.enabled:
            return
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self._ev.append((name, e, time.perf_counter()))

    def finish(self, profile_dir, filename, had_device=1):
        if not self.enabled or len(self._ev) < 2:
            return
        torch.cuda.synchronize()
        rows = []
        for (n0, e0, t0), (_, e1, _) in zip(self._ev[:-1], self._ev[1:]):
            ms = e0.elapsed_time(e1)
            rows.append([n0, t0, t0 + ms / 1e3, ms / 1e3, had_device])
        os.makedirs(profile_dir, exist_ok=True)
        with open(os.path.join(profile_dir, filename), "w", newline="") as fp:
            w = csv.writer(fp)
            w.writerow(["phase", "start_time", "end_time", "elapsed_seconds", "had_device_C"])
            w.writerows(rows)


# ---------------------------------------------------------------------------
# public API
# ---------------------------------------------------------------------------
_PLAN_POOL: dict = {}
_POOL_PER_KEY = 2


class _Lease:
    """Marks a pooled plan busy for as long as this object is alive."""


def _lease_plan(N, M, Lb, steps, weights, owner) -> Plan:
    """A plan for this geometry that no live owner is using, from the pool
    (device workspace is allocated once per shape, not per call)."""
    import weakref
    st, w = normalize_steps(steps, weights)
    key = (torch.cuda.current_device(), N, M, Lb, st.tobytes(), w.tobytes())
    pool = _PLAN_POOL.setdefault(key, [])
    for p in pool:
        if getattr(p, "_lease", None) is None or p._lease() is None:
            p._lease = weakref.ref(owner)
            return p
    p = Plan(N, M, Lb, st, w)
    p._lease = weakref.ref(owner)
    if len(pool) < _POOL_PER_KEY:
        pool.append(p)
    return p


def clear_plan_cache():
    """Release every pooled plan's device memory."""
    for pool in _PLAN_POOL.values():
        for p in pool:
            p.close()
    _PLAN_POOL.clear()


def _buffer_global(L1, L2, beta):
    return min(L1, L2) * (1 - (1 - beta) * min(L1, L2) / max(L1, L2))


def parflex(C, steps, weights, beta, L=None, profile_dir="Profiling_results",
            backtrace_segments=False, warn_slow_chunks=False, slow_chunk_seconds=1.0,
            use_gpu=None):
    """End-to-end ParFlex on a precomputed cost matrix.

    ``C`` is a host array or a CUDA tensor (N x M).  Returns
    ``(best_cost, wp)`` with ``wp`` an int64 (2, K) array, row 0 indexing the
    first sequence (Parflex.py:1510-1547).  Raises ``ValueError`` with the
    reference's message when no endpoint qualifies.
    """
    _require_gpu(use_gpu)
    if L is None:
        L = DEFAULT_CHUNK_LENGTH
    L1, L2 = (int(C.shape[0]), int(C.shape[1]))
    ph = _Phases(profile_dir is not None)
    ph.mark("gpu_host_to_device_C")
    C_dev = cost_matrix_to_gpu(C)
    lease = _Lease()
    plan = _lease_plan(L1, L2, int(L), steps, weights, lease)
    ph.mark("stage1_chunk_flexdtw_all_tiles")
    plan.stage1(C_dev)
    ph.mark("propagate_tile_edge_costs_total")
    plan.propagate(C_dev)
    ph.mark("stage2_scan_and_stitch_total")
    plan.scan(beta)
    plan.stitch()
    ph.mark("end")
    best, end, found, n = plan.result()
    wp = plan.path(n)
    ph.finish(profile_dir, "parflex_end_to_end_phases.csv")
    if warn_slow_chunks:
        warnings.warn("per-chunk timing is not available: all tiles run in one launch")
    if wp.shape[0] == 0:
        return best, np.array([[], []], dtype=np.int64)
    return best, np.ascontiguousarray(wp.T)


def run_flexdtw_on_tiles(C, L, steps=None, weights=None, buffer=1,
                         profile_dir="Profiling_results", warn_slow_chunks=False,
                         slow_chunk_seconds=1.0, use_gpu=None, C_dev=None):
    """Stage 1 on every tile (Parflex_gpu.py:342-607).

    Returns ``(chunks_dict, L, n_chunks_1, n_chunks_2)``; ``chunks_dict`` is a
    read-only mapping keyed by ``(i, j)`` whose values carry the reference's
    keys, materialised lazily from the device.
    """
    _require_gpu(use_gpu)
    if steps is None:
        steps = [(1, 1), (1, 2), (2, 1)]
    if weights is None:
        weights = [2, 3, 3]
    if C is None:
        if C_dev is None:
            raise ValueError("run_flexdtw_on_tiles: provide NumPy C and/or C_dev (both None)")
        L1, L2 = int(C_dev.shape[0]), int(C_dev.shape[1])
    else:
        L1, L2 = C.shape
        if C_dev is not None and tuple(C.shape) != tuple(C_dev.shape):
            raise ValueError("C_dev shape must match C")
    Cd = cost_matrix_to_gpu(C_dev if C_dev is not None else C)
    return _stage1(L1, L2, int(L), steps, weights, profile_dir,
                   lambda plan: plan.stage1(Cd), _CostSource(C_dev=Cd))


def _stage1(L1, L2, Lb, steps, weights, profile_dir, load_and_run, cost):
    holder = _Lease()
    plan = _lease_plan(L1, L2, Lb, steps, weights, holder)
    ph = _Phases(profile_dir is not None)
    ph.mark("stage1_chunk_flexdtw_all_tiles")
    load_and_run(plan)
    ph.mark("end")
    ph.finish(profile_dir, "stage1_runtime_breakdown.csv")
    chunks = ChunksDict(plan, cost)
    chunks._lease_holder = holder  # the plan stays leased while chunks_dict lives
    return chunks, Lb, plan.n1, plan.n2


def tiled_stage1_from_features(F1, F2, steps=None, weights=None, beta=0.1, L=None,
                               use_gpu=None):
    """Features -> cost matrix -> stage 1, all on the device
    (Parflex_gpu.py:610-653).  Returns ``(None, tiled_result)``: like the
    reference's GPU path, C stays on the device in ``tiled_result['C_dev']``."""
    _require_gpu(use_gpu)
    if L is None:
        L = DEFAULT_CHUNK_LENGTH
    f1 = _features_to_device(F1)
    f2 = _features_to_device(F2)
    if f1.dim() != 2 or f2.dim() != 2 or f1.shape[0] != f2.shape[0]:
        raise ValueError("features must be (d, frames) with the same d")
    steps = steps if steps is not None else _STD_STEPS
    weights = weights if weights is not None else np.array([1.25, 3.0, 3.0])
    steps_arr = np.array(steps).reshape((-1, 2))
    stage1_params = {"steps": steps_arr, "weights": np.array(weights), "buffer": 1.0}
    N, M = int(f1.shape[1]), int(f2.shape[1])
    cost = _CostSource(F1=f1, F2=f2)

    def load_and_run(plan):
        plan.load_features(f1, f2)
        plan.stage1()

    chunks, L_out, n1, n2 = _stage1(N, M, int(L), steps, weights, None, load_and_run, cost)
    tiled_result = TiledResult({
        "C_shape": (int(N), int(M)),
        "L_block": L_out,
        "hop": L_out - 1,
        "n_row": n1,
        "n_col": n2,
        "blocks": _blocks(chunks),
        "C": None,
        "stage1_params": stage1_params,
        "chunks_dict": chunks,
        "C_dev": cost,
    })
    return None, tiled_result


class Stage2Result(Mapping):
    """``run_stage2_from_tiled`` result (Parflex.py:1342-1356 keys).  Scalars
    and the stitched path are host values; the slot arrays, edge summary and
    per-segment data copy from the device on first access."""

    _KEYS = ("D_arr", "L_arr", "edge_lens", "best_cost", "best_end", "stitched_wp",
             "n_row", "n_col", "edge_summary", "best_per_segment", "paths_per_segment")

    def __init__(self, plan, eager, backtrace_segments):
        self._plan = plan
        self._d = dict(eager)
        self._bt = backtrace_segments

    def __getitem__(self, k):
        if k not in self._KEYS:
            raise KeyError(k)
        if k not in self._d:
            self._materialise(k)
        return self._d[k]

    def __iter__(self):
        return iter(self._KEYS)

    def __len__(self):
        return len(self._KEYS)

    def _materialise(self, k):
        p = self._plan
        if k == "D_arr":
            self._d[k] = p.host("D_ARR")
        elif k == "L_arr":
            self._d[k] = p.host("L_ARR")
        elif k == "edge_lens":
            el = np.zeros((p.n1, p.n2, 2), np.int64)
            for i in range(p.n1):
                for j in range(p.n2):
                    el[i, j, 0] = min(j * p.hop + p.L, p.M) - j * p.hop
                    el[i, j, 1] = min(i * p.hop + p.L, p.N) - i * p.hop
            self._d[k] = el
        elif k == "edge_summary":
            tD, tL = p.host("TOP_D"), p.host("TOP_L")
            rD, rL = p.host("RIGHT_D"), p.host("RIGHT_L")

            def norm(Dv, Lv):
                out = np.full(Dv.shape, np.nan)
                m = (Lv > 0) & np.isfinite(Dv)
                out[m] = Dv[m] / Lv[m]
                return out
            self._d[k] = {"top": {"D": tD, "L": tL, "norm": norm(tD, tL)},
                          "right": {"D": rD, "L": rL, "norm": norm(rD, rL)}}
        elif k in ("best_per_segment", "paths_per_segment"):
            self._segments()

    def _segments(self):
        p = self._plan
        sn = p.host("SEG_NORM")
        sm = p.host("SEG_META")
        n_top = (p.M + p.L - 1) // p.L
        n_right = (p.N + p.L - 1) // p.L
        names = ["top", "right"]
        bps = {}
        for et in range(2):
            for si in range(n_top if et == 0 else n_right):
                m = sm[et, si]
                if m[0] < 0:
                    continue
                key = (names[et], si)
                bps[key] = {"chunk_i": int(m[0]), "chunk_j": int(m[1]), "edge": int(m[2]),
                            "idx": int(m[3]), "norm_cost": float(sn[et, si]),
                            "global_coord": (int(m[4]), int(m[5])), "segment": key}
        self._d["best_per_segment"] = bps
        paths = {}
        if self._bt:
            for key, meta in bps.items():
                p.stitch((meta["chunk_i"], meta["chunk_j"], meta["edge"], meta["idx"]))
                _, _, _, n = p.result(raise_no_endpoint=False)
                pts = p.path(n)
                paths[key] = {"endpoint": meta,
                              "path": [(int(a), int(b)) for a, b in pts]}
            # restore the best path in the plan's output buffer
            p.stitch()
        self._d["paths_per_segment"] = paths


def run_stage2_from_tiled(tiled_result, C=None, beta=0.1, show_fig=False, top_k=1,
                          profile_dir=None, backtrace_segments=False):
    """Stage 2 on the device (Parflex_gpu.py:857-910): propagation, overlap
    sync, global edge scan and stitched backtrace.  Reads
    ``tiled_result['C_dev']`` when ``C`` is omitted."""
    chunks = tiled_result["chunks_dict"]
    if not isinstance(chunks, ChunksDict):
        raise ValueError("tiled_result was not produced by parflexdtw_b200")
    plan = chunks.plan
    if C is None:
        L1, L2 = tiled_result["C_shape"]
        C_dev = None  # overlap costs come from the plan's own copy of C
    else:
        L1, L2 = C.shape
        C_dev = cost_matrix_to_gpu(C)
    if (int(L1), int(L2)) != (plan.N, plan.M):
        raise ValueError("C shape does not match the stage-1 result")
    if show_fig:
        warnings.warn("show_fig: plotting is not part of parflexdtw_b200")
    ph = _Phases(profile_dir is not None)
    ph.mark("propagate_tile_edge_costs_total")
    plan.propagate(C_dev)
    ph.mark("stage2_scan_and_stitch_total")
    plan.scan(beta)
    plan.stitch()
    ph.mark("end")
    best, end, found, n = plan.result()
    wp = plan.path(n)
    ph.finish(profile_dir, "stage_2_backtrace_compatible.csv")
    eager = {"best_cost": float(best), "best_end": tuple(end),
             "stitched_wp": wp if wp.shape[0] else np.zeros((0, 2), dtype=int),
             "n_row": tiled_result["n_row"], "n_col": tiled_result["n_col"]}
    return Stage2Result(plan, eager, backtrace_segments)


def buffer_global(L1, L2, beta):
    """``min(L1,L2) * (1 - (1-beta) * min(L1,L2) / max(L1,L2))`` (Parflex.py:1520)."""
    return _buffer_global(L1, L2, beta)


__all__ = [
    "DEFAULT_CHUNK_LENGTH", "parflex", "tiled_stage1_from_features",
    "run_stage2_from_tiled", "run_flexdtw_on_tiles", "flexdtw", "flexdtw_chunk_from_global_C",
    "cost_matrix_from_features_gpu", "cost_matrix_to_gpu", "cost_matrix_to_gpu_f32",
    "is_gpu_available", "buffer_global", "ChunksDict", "Stage2Result", "Plan",
    "TiledResult", "clear_plan_cache",
]
