"""Learned tile pruning: a small CNN proposes which L x L tiles the optimal
path crosses, stage 1 runs only on those (and a ring around them), and the
full-tile method is the fallback.

The network reads the cost matrix average-pooled 16x16 (from 16-frame means
of the normalised features: the pooled map of a bilinear cost, no full C),
double centred (row and column means removed) and standardised:

    conv3x3(1 -> 32, stride 4) + ReLU
    conv3x3(32 -> 32, stride 2) + ReLU
    conv3x3(32 -> 1, stride 1)           -> logits, 128 frames per pixel

A tile's score is the max logit over its region.  Training (hand-written
forward / backward / Adam kernels of csrc/cnn.cu, driven from here) uses
labels that the full method itself produces: a tile is positive when the
stitched path of the full-tile FP64 run has a point in it.  Inference keeps
the tiles scoring above a threshold, dilated by one tile (4- or
8-neighbourhood, the one the threshold was calibrated for); when the pruned
run's path comes within 64 to 128 cells of a pruned tile (or no endpoint
qualifies) the full-tile method runs instead.  No counterpart in the reference.

torch supplies device memory only; every computation is a library kernel.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np
import torch

from . import _lib
from .plan import Plan, current_stream_ptr

POOL = 16
CH = 32
STRIDES = (4, 2, 1)
FPP = POOL * STRIDES[0] * STRIDES[1]  # frames per logit pixel
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                               "proposer_L2000.npz")


def _p(t):
    return ct.c_void_p(t.data_ptr()) if t is not None else ct.c_void_p(0)


def tiles_on_path(wp, N, M, L):
    """(n1, n2) uint8: tiles holding a point of the path wp ((K, 2) or (2, K))."""
    wp = np.asarray(wp)
    if wp.shape[0] == 2 and wp.shape[1] != 2:
        wp = wp.T
    hop = L - 1
    n1, n2 = -(-(N - 1) // hop), -(-(M - 1) // hop)
    lab = np.zeros((n1, n2), np.uint8)
    r, c = wp[:, 0], wp[:, 1]
    for di in (0, -1):  # a point on an overlap row belongs to both tiles
        i = np.clip(r // hop + di, 0, n1 - 1)
        okr = (r >= i * hop) & (r < i * hop + L)
        for dj in (0, -1):
            j = np.clip(c // hop + dj, 0, n2 - 1)
            ok = okr & (c >= j * hop) & (c < j * hop + L)
            lab[i[ok], j[ok]] = 1
    return lab


class TileProposer:
    """The proposal network: parameters on the device, kernels from the C ABI."""

    NAMES = ("w1", "b1", "w2", "b2", "w3", "b3")

    def __init__(self, params=None, threshold=0.0, seed=0, device=None, manhattan=False):
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None
                                   else device)
        self.threshold = float(threshold)
        self.manhattan = bool(manhattan)  # dilation the threshold was calibrated for
        if params is None:
            g = torch.Generator().manual_seed(seed)
            shapes = {"w1": (CH, 1, 3, 3), "w2": (CH, CH, 3, 3), "w3": (1, CH, 3, 3)}
            params = {}
            for k, shp in shapes.items():
                fan_in = shp[1] * 9
                params[k] = torch.randn(shp, generator=g) * np.sqrt(2.0 / fan_in)
            params["b1"] = torch.zeros(CH)
            params["b2"] = torch.zeros(CH)
            params["b3"] = torch.full((1,), -2.0)
        self.params = {k: torch.as_tensor(np.asarray(params[k]), dtype=torch.float32)
                       .to(self.device).contiguous() for k in self.NAMES}

    # -- persistence -------------------------------------------------------
    def save(self, path, **meta):
        np.savez(path, threshold=self.threshold, manhattan=self.manhattan,
                 strides=np.asarray(STRIDES),
                 **{k: v.cpu().numpy() for k, v in self.params.items()}, **meta)

    @classmethod
    def load(cls, path=DEFAULT_WEIGHTS):
        z = np.load(path)
        if "strides" not in z or tuple(int(x) for x in z["strides"]) != STRIDES:
            raise ValueError(f"{path}: weights for another network layout")
        return cls({k: z[k] for k in cls.NAMES}, threshold=float(z["threshold"]),
                   manhattan=bool(z["manhattan"]))

    # -- building blocks ---------------------------------------------------
    @staticmethod
    def pooled_cost(f1, f2, center=True):
        """16x average-pooled cost matrix (P1 x P2, FP32) of device features
        (d x N, d x M, FP64); with center (the network's input), double
        centred and standardised (pfx_pooled_center)."""
        lib = _lib.load()
        s = current_stream_ptr()
        d, N = f1.shape
        M = f2.shape[1]
        P1, P2 = -(-N // POOL), -(-M // POOL)
        A = torch.empty((d, P1), dtype=torch.float32, device=f1.device)
        B = torch.empty((d, P2), dtype=torch.float32, device=f1.device)
        out = torch.empty((P1, P2), dtype=torch.float32, device=f1.device)
        _lib.check(lib.pfx_pool_features(_p(f1), d, N, POOL, _p(A), s))
        _lib.check(lib.pfx_pool_features(_p(f2), d, M, POOL, _p(B), s))
        _lib.check(lib.pfx_pooled_cost(_p(A), _p(B), d, P1, P2, _p(out), s))
        if center:
            sc = torch.empty(P1 + P2 + 2, dtype=torch.float32, device=f1.device)
            _lib.check(lib.pfx_pooled_center(_p(out), P1, P2, _p(sc), s))
        return out

    def forward(self, pooled, keep=False, bf16=False):
        """Logits (H3 x W3) of one pooled map; with keep, also the layer
        inputs and outputs for backward.  bf16: store the hidden activations
        in bf16 (inference)."""
        lib = _lib.load()
        s = current_stream_ptr()
        H, W = pooled.shape
        x = pooled.contiguous()
        acts = [x]
        cin = 1
        layers = ((self.params["w1"], self.params["b1"], CH, STRIDES[0], 1),
                  (self.params["w2"], self.params["b2"], CH, STRIDES[1], 1),
                  (self.params["w3"], self.params["b3"], 1, STRIDES[2], 0))
        x_bf = 0
        for li, (w, b, cout, st, relu) in enumerate(layers):
            Ho, Wo = (H - 1) // st + 1, (W - 1) // st + 1
            y_bf = 1 if (bf16 and li < 2) else 0
            y = torch.empty((cout, Ho, Wo), dtype=torch.bfloat16 if y_bf else torch.float32,
                            device=pooled.device)
            _lib.check(lib.pfx_conv3x3_forward(_p(x), x_bf, cin, H, W, _p(w), _p(b), cout, st,
                                               relu, _p(y), y_bf, s))
            acts.append(y)
            x, x_bf, cin, H, W = y, y_bf, cout, Ho, Wo
        logits = x.reshape(H, W)
        return (logits, acts) if keep else logits

    @staticmethod
    def tile_scores(logits, N, M, L):
        lib = _lib.load()
        hop = L - 1
        n1, n2 = -(-(N - 1) // hop), -(-(M - 1) // hop)
        H, W = logits.shape
        score = torch.empty(n1 * n2, dtype=torch.float32, device=logits.device)
        arg = torch.empty(n1 * n2, dtype=torch.int32, device=logits.device)
        _lib.check(lib.pfx_tile_max(_p(logits), H, W, n1, n2, hop, L, N, M, FPP, _p(score),
                                    _p(arg), current_stream_ptr()))
        return score, arg, (n1, n2)

    # -- inference into preallocated buffers (graph-capturable) ---------------
    @staticmethod
    def buffers(d, N, M, L, device):
        """Device buffers of one proposer pass for pairs of up to N x M frames
        at tile length L (every kernel takes its sizes explicitly, so a set
        sized for the largest pair serves any smaller one)."""
        P1, P2 = -(-N // POOL), -(-M // POOL)
        H, W = P1, P2
        dims = []
        for st in STRIDES:
            H, W = (H - 1) // st + 1, (W - 1) // st + 1
            dims.append((H, W))
        hop = L - 1
        nt = -(-(N - 1) // hop) * -(-(M - 1) // hop)
        f32, bf = dict(dtype=torch.float32, device=device), dict(dtype=torch.bfloat16,
                                                                 device=device)
        mom = int(_lib.load().pfx_pooled_center_scratch(P1, P2))
        return {"A": torch.empty(d * P1, **f32), "B": torch.empty(d * P2, **f32),
                "mom": torch.empty(max(mom, 8), dtype=torch.uint8, device=device),
                "y1": torch.empty(CH * dims[0][0] * dims[0][1], **bf),
                "y2": torch.empty(CH * dims[1][0] * dims[1][1], **bf),
                "y3": torch.empty(dims[2][0] * dims[2][1], **f32),
                "score": torch.empty(max(nt, 1), **f32),
                "arg": torch.empty(max(nt, 1), dtype=torch.int32, device=device)}

    def propose_into(self, f1, f2, L, bufs, mask, threshold=None, dilation=1, manhattan=None):
        """The inference of ``propose`` from device features (d x N, d x M,
        FP64) into preallocated ``bufs`` (``buffers``), writing the tile mask
        into the uint8 device tensor ``mask`` (n1 * n2 entries).  Launches
        only library kernels on the current stream, allocates nothing.

        The network's centred, standardised input is never stored: the pooled
        features are centred and scaled (``pfx_pooled_center_features``) so
        that their product is that map, and the first layer computes it per
        input patch (``pfx_conv3x3_forward_features``).  In real arithmetic
        this is the input ``propose`` builds; FP32 rounding differs."""
        lib = _lib.load()
        s = current_stream_ptr()
        d, N = int(f1.shape[0]), int(f1.shape[1])
        M = int(f2.shape[1])
        if d > 16:
            raise ValueError("propose_into takes d <= 16 features (use propose)")
        P1, P2 = -(-N // POOL), -(-M // POOL)
        _lib.check(lib.pfx_pool_features(_p(f1), d, N, POOL, _p(bufs["A"]), s))
        _lib.check(lib.pfx_pool_features(_p(f2), d, M, POOL, _p(bufs["B"]), s))
        _lib.check(lib.pfx_pooled_center_features(_p(bufs["A"]), _p(bufs["B"]), d, P1, P2,
                                                  _p(bufs["mom"]), s))
        w, b = self.params["w1"], self.params["b1"]
        _lib.check(lib.pfx_conv3x3_forward_features(_p(bufs["A"]), _p(bufs["B"]), d, P1, P2,
                                                    _p(w), _p(b), CH, STRIDES[0], 1,
                                                    _p(bufs["y1"]), 1, s))
        H, W = (P1 - 1) // STRIDES[0] + 1, (P2 - 1) // STRIDES[0] + 1
        x, x_bf, cin = bufs["y1"], 1, CH
        layers = ((self.params["w2"], self.params["b2"], CH, STRIDES[1], 1, bufs["y2"], 1),
                  (self.params["w3"], self.params["b3"], 1, STRIDES[2], 0, bufs["y3"], 0))
        for w, b, cout, st, relu, y, y_bf in layers:
            Ho, Wo = (H - 1) // st + 1, (W - 1) // st + 1
            _lib.check(lib.pfx_conv3x3_forward(_p(x), x_bf, cin, H, W, _p(w), _p(b), cout, st,
                                               relu, _p(y), y_bf, s))
            x, x_bf, cin, H, W = y, y_bf, cout, Ho, Wo
        hop = L - 1
        n1, n2 = -(-(N - 1) // hop), -(-(M - 1) // hop)
        _lib.check(lib.pfx_tile_max(_p(x), H, W, n1, n2, hop, L, N, M, FPP, _p(bufs["score"]),
                                    _p(bufs["arg"]), s))
        thr = self.threshold if threshold is None else float(threshold)
        manhattan = self.manhattan if manhattan is None else manhattan
        _lib.check(lib.pfx_tile_mask_from_scores(_p(bufs["score"]), n1, n2, thr, int(dilation),
                                                 int(bool(manhattan)), _p(mask), s))

    def propose(self, pooled, N, M, L, threshold=None, dilation=1, manhattan=None):
        """Device uint8 mask (n1 x n2) of the tiles to run, and the scores:
        tiles above the threshold, dilated by `dilation` tiles (Chebyshev
        distance, or Manhattan with `manhattan`)."""
        logits = self.forward(pooled, bf16=True)
        score, _, (n1, n2) = self.tile_scores(logits, N, M, L)
        mask = torch.empty(n1 * n2, dtype=torch.uint8, device=pooled.device)
        thr = self.threshold if threshold is None else float(threshold)
        manhattan = self.manhattan if manhattan is None else manhattan
        _lib.check(_lib.load().pfx_tile_mask_from_scores(_p(score), n1, n2, thr, int(dilation),
                                                         int(bool(manhattan)), _p(mask),
                                                         current_stream_ptr()))
        return mask.reshape(n1, n2), score.reshape(n1, n2)

    # -- training ------------------------------------------------------------
    def init_optimizer(self):
        self.opt = {k: (torch.zeros_like(v), torch.zeros_like(v)) for k, v in self.params.items()}
        self.opt_step = 0

    def gradients(self, pooled, label, N, M, L, pos_weight):
        """(loss, grads dict) for one map and its (n1, n2) tile labels."""
        lib = _lib.load()
        s = current_stream_ptr()
        logits, acts = self.forward(pooled, keep=True)
        score, arg, (n1, n2) = self.tile_scores(logits, N, M, L)
        lab = torch.as_tensor(np.ascontiguousarray(label, dtype=np.uint8).reshape(-1),
                              device=pooled.device)
        loss = torch.zeros(1, dtype=torch.float32, device=pooled.device)
        dscore = torch.empty_like(score)
        _lib.check(lib.pfx_tile_bce(_p(score), _p(lab), n1 * n2, float(pos_weight), _p(loss),
                                    _p(dscore), s))
        dy = torch.zeros_like(logits)
        _lib.check(lib.pfx_tile_max_backward(_p(dscore), _p(arg), n1 * n2, _p(dy), s))
        grads = {k: torch.zeros_like(v) for k, v in self.params.items()}
        layers = ((1, CH, STRIDES[0], 1), (CH, CH, STRIDES[1], 1), (CH, 1, STRIDES[2], 0))
        dy = dy.reshape(1, *logits.shape)
        for li in (2, 1, 0):
            cin, cout, st, relu = layers[li]
            x, y = acts[li], acts[li + 1]
            H, W = x.shape[-2:]
            dx = torch.empty((cin, H, W), dtype=torch.float32, device=x.device) if li else None
            _lib.check(lib.pfx_conv3x3_backward(
                _p(x), cin, H, W, _p(self.params[f"w{li + 1}"]), cout, st, _p(y), relu, _p(dy),
                _p(dx), _p(grads[f"w{li + 1}"]), _p(grads[f"b{li + 1}"]), s))
            dy = dx
        return loss, grads

    def step(self, grads, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        lib = _lib.load()
        s = current_stream_ptr()
        self.opt_step += 1
        for k, p in self.params.items():
            m, v = self.opt[k]
            _lib.check(lib.pfx_adam_step(_p(p), _p(grads[k]), _p(m), _p(v), p.numel(), lr, b1,
                                         b2, eps, self.opt_step, s))


FALLBACK_MARGIN = 64  # cells


def _pruned_near_path(wp, mask, N, M, L, margin=FALLBACK_MARGIN):
    """(n1, n2) bool: the pruned tiles that come within about `margin` cells
    of the path wp.  The test works on margin x margin cell blocks: for every
    block the path touches, the tiles covering a cell of it or of its 8
    neighbouring blocks must all have run (so the distance tested is margin
    to 2 margin cells).  The path is monotone, so per row of blocks it
    touches one interval of blocks, and a summed-area table of the pruned
    tiles answers each interval's rectangle at once."""
    wp = np.asarray(wp)
    if wp.shape[0] == 2 and wp.shape[1] != 2:
        wp = wp.T
    m = np.asarray(mask, bool)
    near = np.zeros(m.shape, bool)
    if m.all() or wp.shape[0] == 0:
        return near
    n1, n2 = m.shape
    hop, B = L - 1, int(margin)
    r, c = wp[:, 0], wp[:, 1]
    a = np.arange(r[0] // B, r[-1] // B + 1)
    st = np.searchsorted(r, a * B, "left")
    en = np.searchsorted(r, (a + 1) * B, "left")
    ok = en > st
    a, st, en = a[ok], st[ok], en[ok]
    r0 = np.maximum(a - 1, 0) * B
    r1 = np.minimum((a + 2) * B, N) - 1
    c0 = np.maximum(c[st] // B - 1, 0) * B
    c1 = np.minimum((c[en - 1] // B + 2) * B, M) - 1
    # tiles i with i*hop <= r1 and i*hop + L - 1 >= r0
    ilo = np.clip(-(-(r0 - (L - 1)) // hop), 0, n1 - 1)
    ihi = np.clip(r1 // hop, 0, n1 - 1)
    jlo = np.clip(-(-(c0 - (L - 1)) // hop), 0, n2 - 1)
    jhi = np.clip(c1 // hop, 0, n2 - 1)
    sat = np.zeros((n1 + 1, n2 + 1), np.int64)
    sat[1:, 1:] = np.cumsum(np.cumsum(~m, axis=0), axis=1)
    cnt = sat[ihi + 1, jhi + 1] - sat[ilo, jhi + 1] - sat[ihi + 1, jlo] + sat[ilo, jlo]
    for k in np.flatnonzero(cnt > 0):
        near[ilo[k]:ihi[k] + 1, jlo[k]:jhi[k] + 1] = True
    return near & ~m


def _needs_fallback(wp, mask, N, M, L, margin=FALLBACK_MARGIN):
    """True when the path comes within about `margin` cells of a pruned
    tile's cells: there it may have been cut off (_pruned_near_path)."""
    return bool(_pruned_near_path(wp, mask, N, M, L, margin).any())


def parflex_pruned(F1, F2, steps, weights, beta, L, proposer=None, threshold=None,
                   dilation=1, precision="fp64", plan=None, warps=None):
    """ParFlex from features with learned tile pruning.

    Returns ``(best_cost, wp[2, K], info)``; ``info`` has the tile counts, the
    skipped fraction and whether the full-tile fallback ran (and why).
    """
    from .parflex import _features_to_device
    f1 = _features_to_device(F1)
    f2 = _features_to_device(F2)
    N, M = int(f1.shape[1]), int(f2.shape[1])
    if proposer is None:
        proposer = TileProposer.load()
    own = plan is None
    if own:
        plan = Plan(N, M, L, steps, weights, precision=precision)
    pooled = proposer.pooled_cost(f1, f2)
    mask, _ = proposer.propose(pooled, N, M, L, threshold, dilation)
    m_host = mask.cpu().numpy()
    kept = int(m_host.sum())
    total = plan.n1 * plan.n2
    info = {"tiles_total": total, "tiles_run": kept, "skipped_fraction": 1 - kept / total,
            "fallback": False, "reason": None}
    full_warps = plan.warps
    best = wp = None
    if kept:
        plan.set_tile_mask(mask)
        if warps or kept < 2 * 148:
            plan.set_warps(warps or 16)
        plan.load_features(f1, f2)
        plan.run(None, beta)
        try:
            best, end, found, n = plan.result()
            wp = plan.path(n)
            if _needs_fallback(wp, m_host, N, M, L):
                info.update(fallback=True, reason="path near a pruned tile")
        except ValueError:
            info.update(fallback=True, reason="no endpoint among proposed tiles")
    else:
        info.update(fallback=True, reason="no tile proposed")
    if info["fallback"]:
        plan.set_tile_mask(None)
        plan.set_warps(full_warps)
        plan.load_features(f1, f2)
        plan.run(None, beta)
        best, end, found, n = plan.result()
        wp = plan.path(n)
        info["tiles_run"] = kept + total
    else:
        plan.set_tile_mask(None)
        plan.set_warps(full_warps)
    return best, np.ascontiguousarray(wp.T), info


class PrunedBatch:
    """Learned pruning over a batch of pairs: one proposer pass per pair,
    then the kept tiles of all pairs in one stage-1 launch per wave
    (``pfx_batch_set_masks``), stage 2 per pair.  A pair whose path comes
    near a pruned tile gets those tiles added and runs again (up to `expand`
    times; ``pfx_batch_complete``: stage 1 only on the added tiles); a pair
    still near one, or without an endpoint, falls back to the full-tile
    method (every tile not run yet)."""

    def __init__(self, shapes, L, steps, weights, d, proposer=None, threshold=None,
                 dilation=1, manhattan=None, precision="fp64", wave_bytes=0, warps=0,
                 expand=2, cost="slabs", proposer_streams=8, cost_fma=False):
        from .batch import Batch
        self.batch = Batch(shapes, L, steps, weights, d, wave_bytes=wave_bytes, warps=warps,
                           precision=precision, cost=cost, cost_fma=cost_fma)
        self.proposer = proposer or TileProposer.load()
        self.threshold = threshold
        self.dilation = dilation
        self.manhattan = manhattan
        self.expand = int(expand)
        self.proposer_streams = int(proposer_streams)
        self._streams = None
        self._graph = None
        self.L = int(L)
        self.steps, self.weights, self.precision = steps, weights, precision
        self.shapes = [(int(n), int(m)) for n, m in shapes]
        hop = self.L - 1
        self.grids = [(-(-(n - 1) // hop), -(-(m - 1) // hop)) for n, m in self.shapes]
        self.offs = np.concatenate([[0], np.cumsum([a * b for a, b in self.grids])])

    def load(self, pairs, non_blocking=True):
        self.batch.load(pairs, non_blocking=non_blocking)

    def run(self, beta, profile=False, host_pairs=None):
        """[(best_cost, wp[2, K]) per pair], info.  profile: synchronise
        between phases and report their wall times (ms) in info.

        host_pairs: the pairs' features as page-locked host tensors (d x N,
        d x M, float64), uploaded as part of the run: each pair's upload runs
        on the proposer stream of that pair, just before its proposer pass, so
        that it overlaps the other pairs' passes (the phase, uploads included,
        is recorded once per set of host buffers into a CUDA graph).  Without
        it the features are the ones ``load`` put on the device."""
        import time as _time
        b = self.batch
        marks = []

        def mark(name):
            if profile:
                torch.cuda.synchronize()
                marks.append((name, _time.perf_counter()))

        mark("start")
        masks = self._propose_all(host_pairs)
        mark("proposer")
        self.last_masks = masks  # the proposed tiles, pairs' (n1, n2) masks concatenated
        b.set_masks(masks)
        mark("set_masks")
        b.run(beta, use_graph=False)
        mark("align")
        align_ms = b.timing() if profile else None
        near_d, flags_d = b.check_paths(FALLBACK_MARGIN)
        best, end, lens = b.results()
        flags = flags_d.cpu().numpy()
        paths = b.paths_rows(lens)
        mark("results")
        out, fallbacks, reasons, expanded = [], 0, {}, 0
        kept = int(masks.sum())
        run_tiles = kept
        n = len(self.shapes)
        todo = [i for i in range(n) if flags[i] or not end[i, 6]]
        if todo:
            m_host = masks.cpu().numpy()
            near = near_d.cpu().numpy()
        out = [(float(best[i]), paths[i]) for i in range(n)]
        for i in todo:
            N, M = self.shapes[i]
            mk = m_host[self.offs[i]:self.offs[i + 1]].reshape(self.grids[i])
            reason = "no endpoint among proposed tiles" if not end[i, 6] \
                else "path near a pruned tile"
            if reason == "path near a pruned tile" and self.expand > 0:
                add = near[self.offs[i]:self.offs[i + 1]].reshape(self.grids[i]).astype(bool)
                res, ran = self._expand(i, N, M, beta, add, mk)
                if res is not None:
                    expanded += 1
                    run_tiles += ran
                    out[i] = res
                    continue
            # the full-tile method: every tile not run yet
            fallbacks += 1
            reasons[reason] = reasons.get(reason, 0) + 1
            bc, wp = self._full(i, N, M, beta)
            out[i] = (bc, np.ascontiguousarray(wp.T))
            run_tiles += self.grids[i][0] * self.grids[i][1] - int(mk.sum())
        mark("checks")
        total = int(self.offs[-1])
        info = {"tiles_total": total, "tiles_run": run_tiles, "tiles_proposed": kept,
                "skipped_fraction": 1 - kept / total, "fallbacks": fallbacks,
                "fallback_reasons": reasons, "expanded": expanded, "waves": b.waves}
        if profile:
            info["phases_ms"] = {marks[k][0]: 1e3 * (marks[k][1] - marks[k - 1][1])
                                 for k in range(1, len(marks))}
            info["align_ms"] = dict(zip(("cost", "stage1", "stage2"), align_ms))
        return out, info

    def _launch_proposer(self, host=None):
        """Every pair's proposer pass, pairs spread over the side streams
        (the kernels are small), each stream with its own buffer set; with
        `host` ((F1, F2) page-locked host tensors per pair), each pair's
        upload first, on the same stream."""
        main = torch.cuda.current_stream()
        lib = _lib.load()
        for st in self._streams:
            st.wait_stream(main)  # features loaded (or their buffers free)
        for i, (N, M) in enumerate(self.shapes):
            k = i % len(self._streams)
            with torch.cuda.stream(self._streams[k]):
                if host is not None:
                    h1, h2 = host[i]
                    _lib.check(lib.pfx_batch_load_async(
                        self.batch.handle, i, ct.c_void_p(h1.data_ptr()),
                        ct.c_void_p(h2.data_ptr()), current_stream_ptr()))
                f1, f2 = self._views[i]
                self.proposer.propose_into(f1, f2, self.L, self._bufs[k],
                                           self._masks[self.offs[i]:self.offs[i + 1]],
                                           self.threshold, self.dilation, self.manhattan)
        for st in self._streams:
            main.wait_stream(st)

    def _setup_proposer(self):
        dev = self.proposer.device
        self._masks = torch.empty(int(self.offs[-1]), dtype=torch.uint8, device=dev)
        self._views = [self.batch.feature_views(i) for i in range(len(self.shapes))]
        ns = max(1, min(self.proposer_streams, len(self.shapes)))
        self._streams = [torch.cuda.Stream(device=dev) for _ in range(ns)]
        self._bufs = []
        for k in range(ns):
            mine = self.shapes[k::ns]
            self._bufs.append(TileProposer.buffers(self.batch.d, max(n for n, _ in mine),
                                                   max(m for _, m in mine), self.L, dev))
        self._host_graphs = {}

    def _check_host(self, host_pairs):
        if len(host_pairs) != len(self.shapes):
            raise ValueError(f"{len(host_pairs)} pairs for a batch of {len(self.shapes)}")
        out = []
        for i, (F1, F2) in enumerate(host_pairs):
            for t, n in ((F1, self.shapes[i][0]), (F2, self.shapes[i][1])):
                if not (isinstance(t, torch.Tensor) and t.device.type == "cpu" and t.is_pinned()
                        and t.dtype == torch.float64 and t.is_contiguous()):
                    raise ValueError("host_pairs: contiguous page-locked float64 CPU tensors "
                                     "(torch.Tensor.pin_memory())")
                if tuple(t.shape) != (self.batch.d, n):
                    raise ValueError(f"pair {i}: features {tuple(t.shape)}, expected "
                                     f"({self.batch.d}, {n})")
            out.append((F1, F2))
        return out

    def _propose_all(self, host_pairs=None):
        """The tile masks of all pairs (uint8 device tensor, pairs' (n1, n2)
        masks concatenated): one eager pass on the first call, which also
        records the whole phase into a CUDA graph; the graph is replayed on
        every later call (the features are read from the batch's fixed
        buffers; with host_pairs, a graph per set of host buffers uploads
        them first)."""
        if self._streams is None:
            self._setup_proposer()
        if host_pairs is not None:
            host = self._check_host(host_pairs)
            key = tuple((a.data_ptr(), c.data_ptr()) for a, c in host)
            g = self._host_graphs.get(key)
            if g is None:
                self._launch_proposer(host)
                torch.cuda.current_stream().synchronize()
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g):
                    self._launch_proposer(host)
                self._host_graphs[key] = (g, host)  # the graph reads these buffers
                return self._masks
            g[0].replay()
            return self._masks
        if self._graph is None:
            self._launch_proposer()
            torch.cuda.current_stream().synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                self._launch_proposer()
            self._graph = g
            return self._masks
        self._graph.replay()
        return self._masks

    def _expand(self, i, N, M, beta, add, mk):
        """Adds `add` (the pruned tiles the path came near) to pair i's run
        and aligns it again (stage 1 only on the added tiles), up to
        `expand` times while the new path stays near pruned tiles.  Returns
        ((best_cost, wp[2, K]) or None when still near, tiles added)."""
        m = np.asarray(mk, bool).copy()
        ran = 0
        for _ in range(self.expand):
            try:
                bc, wp = self.batch.complete(i, beta, add)
            except ValueError as e:
                if str(e) == _lib.NO_ENDPOINT_MSG:
                    return None, ran
                raise
            ran += int(add.sum())
            m |= add
            add = _pruned_near_path(wp, m, N, M, self.L)
            if not add.any():
                return (bc, np.ascontiguousarray(wp.T)), ran
        return None, ran

    def _full(self, i, N, M, beta):
        """The full-tile method for pair i: completed inside the batch when
        the pool holds its slabs (the masked-in tiles' stage 1 is reused),
        else on a plan of its own."""
        try:
            return self.batch.complete(i, beta)
        except ValueError as e:
            if str(e) == _lib.NO_ENDPOINT_MSG or self.batch.cost_fma:
                raise  # (a plan of its own has no FMA-chain cost)
            f1, f2 = self.batch.feature_views(i)
            plan = Plan(N, M, self.L, self.steps, self.weights, precision=self.precision)
            plan.load_features(f1, f2)
            plan.run(None, beta)
            bc, _, _, n = plan.result()
            wp = plan.path(n)
            plan.close()
            return bc, wp

    def close(self):
        self._graph = None
        self._host_graphs = {}
        self.batch.close()
