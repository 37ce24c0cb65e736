"""Autotuner for batched alignment: tile length per length bucket and stage-1
warps per tile CTA.

The tile length L decides how a pair is cut: larger tiles have more 64-row
strips in flight per tile (the strip pipeline of the stage-1 kernel is busy
for nS / (nS - 1 + warps) of its span) and fewer tile edges for stage 2;
smaller tiles give more tiles to spread over the 148 SMs.  Warps per tile
(4, 8, 16 -> 4, 2, 1 tile CTAs per SM) trades the same way.  The tuner times
probe batches of the real shapes of each bucket (seeded synthetic
chroma-like features) with CUDA events for every candidate and keeps the
fastest per bucket; the batch then runs all pairs in one launch per wave
with the warps choice of the bucket holding most of the cells.

Results are cached per (device, bucket, steps, weights, d, precision) in
memory and,
when ``cache_path`` is given, in a JSON file.
"""
from __future__ import annotations

import json
import os

import numpy as np
import torch

from .batch import Batch
from .workloads import warped_pair

CANDIDATE_L = (1000, 2000)
CANDIDATE_WARPS = (4, 8, 16)
BUCKET_EDGES = (4000, 8000, 14000)  # on min(N, M)


class Autotuner:
    def __init__(self, candidates_L=CANDIDATE_L, candidates_warps=CANDIDATE_WARPS,
                 bucket_edges=BUCKET_EDGES, probe_pairs=16, repeats=2, seed=0,
                 cache_path=None):
        self.candidates_L = tuple(int(x) for x in candidates_L)
        self.candidates_warps = tuple(int(x) for x in candidates_warps)
        self.bucket_edges = tuple(int(x) for x in bucket_edges)
        self.probe_pairs = int(probe_pairs)
        self.repeats = int(repeats)
        self.seed = int(seed)
        self.cache_path = cache_path
        self.table = {}
        self.log = []  # (bucket, L, warps, ms per pair) of every probe
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.table = {k: tuple(v) for k, v in json.load(f).items()}

    def bucket(self, N, M) -> int:
        return int(np.searchsorted(self.bucket_edges, min(N, M), side="right"))

    def _key(self, b, steps, weights, d, precision):
        name = torch.cuda.get_device_name() if torch.cuda.is_available() else "none"
        st = np.asarray(steps, dtype=np.int64).reshape(-1).tolist()
        w = np.asarray(weights, dtype=np.float64).reshape(-1).tolist()
        return f"{name}|b{b}|{st}|{w}|d{d}|{precision}"

    def _probe(self, shapes, Lb, warps, steps, weights, d, precision, beta=0.1):
        """Milliseconds per pair of one batch run (graph replay, after warm-up),
        or None when the configuration does not fit."""
        rng = np.random.default_rng(self.seed)
        pairs = [warped_pair(rng, n, m, d=d) for n, m in shapes]
        shapes = [(p[0].shape[1], p[1].shape[1]) for p in pairs]
        try:
            b = Batch(shapes, Lb, steps, weights, d, warps=warps, precision=precision)
        except ValueError:
            return None
        try:
            b.load(pairs)
            b.run(beta)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(self.repeats):
                b.run(beta)
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / self.repeats / len(shapes)
        finally:
            b.close()

    def tune_bucket(self, shapes, steps, weights, d, precision="fp64"):
        """(L, warps) with the least time per pair for these shapes."""
        sel = shapes[:self.probe_pairs]
        best = None
        for Lb in self.candidates_L:
            for w in self.candidates_warps:
                ms = self._probe(sel, Lb, w, steps, weights, d, precision)
                self.log.append((self.bucket(*sel[0]), Lb, w, ms))
                if ms is not None and (best is None or ms < best[2]):
                    best = (Lb, w, ms)
        if best is None:
            raise ValueError("no tile length / warps candidate fits these shapes")
        return best[0], best[1]

    def choose(self, shapes, steps, weights, d, precision="fp64"):
        """Per-pair tile lengths and one warps-per-tile value for a batch."""
        groups = {}
        for i, (n, m) in enumerate(shapes):
            groups.setdefault(self.bucket(n, m), []).append(i)
        Ls = [0] * len(shapes)
        cells = {}
        for b, idx in groups.items():
            key = self._key(b, steps, weights, d, precision)
            if key not in self.table:
                # representative probe shapes: spread over the bucket's pairs
                pick = [shapes[i] for i in idx[::max(1, len(idx) // self.probe_pairs)]]
                self.table[key] = self.tune_bucket(pick, steps, weights, d, precision)
                self._save()
            Lb, w = self.table[key]
            for i in idx:
                Ls[i] = Lb
            cells[b] = sum(shapes[i][0] * shapes[i][1] for i in idx)
        main = max(cells, key=cells.get)
        warps = self.table[self._key(main, steps, weights, d, precision)][1]
        return Ls, warps

    def _save(self):
        if self.cache_path:
            with open(self.cache_path, "w") as f:
                json.dump({k: list(v) for k, v in self.table.items()}, f, indent=1)


_DEFAULT = None


def default_tuner() -> Autotuner:
    global _DEFAULT
    if _DEFAULT is None:
        _DEFAULT = Autotuner()
    return _DEFAULT
