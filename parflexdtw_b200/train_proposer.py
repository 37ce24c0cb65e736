"""Train the tile proposer on pairs the full method labels.

    python -m parflexdtw_b200.train_proposer --pairs 5000 --epochs 6 \\
        --out parflexdtw_b200/data/proposer_L2000.npz

Training pairs: N ~ U(5000, 30000), M = N x U(0.7, 1.4), 12-d chroma-like
features with 0-10 % unrelated padding per end (the warp model of
workloads.warped_pair).  Labels: the tiles (L = 2000) crossed by the stitched
path of the full-tile FP64 method, run in device batches.  The network then
trains with the library's own forward / backward / Adam kernels (batch of
one map, weighted BCE over tiles).  The threshold saved with the weights is
the highest at which, with the one-tile dilation, every labelled tile of a
held-out split is run, minus a margin (one tile of dilation: the
4-neighbourhood by default).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import workloads as W
from .batch import Batch
from .prune import TileProposer, tiles_on_path

STEPS = ((1, 1), (1, 2), (2, 1))
WEIGHTS = (2.0, 3.0, 3.0)


def make_pairs(n, seed, lo=5000, hi=30000, pad=0.1):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        N = int(rng.integers(lo, hi + 1))
        m = int(round(N * rng.uniform(0.7, 1.4)))
        out.append(W.warped_pair(rng, N, m, pad_frac=pad))
    return out


def label_pairs(pairs, L, beta):
    """Tiles crossed by the full-tile FP64 path of every pair (one device
    batch), or None for a pair without an endpoint."""
    b = Batch([(p[0].shape[1], p[1].shape[1]) for p in pairs], L, STEPS, WEIGHTS, 12)
    b.load(pairs)
    b.run(beta, use_graph=False)
    best, end, lens = b.results()
    paths = b.paths(lens)
    b.close()
    return [tiles_on_path(wp, F1.shape[1], F2.shape[1], L) if ok else None
            for (F1, F2), wp, ok in zip(pairs, paths, end[:, 6])]


def build_dataset(n, seed, L, beta, net, chunk=64, log=print):
    """(pooled map on the device, labels, N, M) per pair, generated and
    labelled `chunk` pairs at a time (features are not kept)."""
    data = []
    t0 = time.perf_counter()
    for c0 in range(0, n, chunk):
        pairs = make_pairs(min(chunk, n - c0), seed + c0)
        for (F1, F2), lab in zip(pairs, label_pairs(pairs, L, beta)):
            if lab is None:
                continue
            pooled = net.pooled_cost(torch.from_numpy(F1).cuda(), torch.from_numpy(F2).cuda())
            data.append((pooled, lab, F1.shape[1], F2.shape[1]))
        log(f"labelled {min(c0 + chunk, n)}/{n} pairs ({time.perf_counter() - t0:.1f} s)")
    return data


def train(net, data, L, epochs, lr, log=print, seed=0):
    rng = np.random.default_rng(seed)
    net.init_optimizer()
    pos = sum(int(lab.sum()) for _, lab, _, _ in data)
    tot = sum(lab.size for _, lab, _, _ in data)
    pos_weight = float(min(20.0, (tot - pos) / max(pos, 1)))
    hist = []
    for ep in range(epochs):
        t0 = time.perf_counter()
        order = rng.permutation(len(data))
        acc = torch.zeros(1, device="cuda")
        lr_ep = lr * (0.5 ** (ep // 2))
        for k in order:
            pooled, lab, N, M = data[k]
            loss, g = net.gradients(pooled, lab, N, M, L, pos_weight)
            net.step(g, lr=lr_ep)
            acc += loss
        mean = float(acc.item()) / len(data)
        hist.append(mean)
        log(f"epoch {ep}: loss {mean:.4f} lr {lr_ep:.1e} ({time.perf_counter() - t0:.1f} s)")
    return hist, pos_weight


def calibrate(net, data, L, margin=0.5, manhattan=True):
    """The highest threshold at which, with one tile of dilation (4- or
    8-neighbourhood), every labelled tile of every pair in `data` is run
    (minus a margin); and the fraction of tiles kept at that threshold."""
    thr = np.inf
    for pooled, lab, N, M in data:
        s = net.tile_scores(net.forward(pooled, bf16=True), N, M, L)[0].cpu().numpy()
        s = s.reshape(lab.shape)
        p = np.pad(s, 1, constant_values=-np.inf)
        nb = np.full_like(s, -np.inf)
        for di in range(3):
            for dj in range(3):
                if manhattan and abs(di - 1) + abs(dj - 1) > 1:
                    continue
                nb = np.maximum(nb, p[di:di + s.shape[0], dj:dj + s.shape[1]])
        thr = min(thr, float(nb[lab.astype(bool)].min()))
    thr -= margin
    kept = total = 0
    for pooled, lab, N, M in data:
        mask, _ = net.propose(pooled, N, M, L, thr, 1, manhattan)
        kept += int(mask.sum().item())
        total += lab.size
    return thr, kept / total


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=5000)
    ap.add_argument("--val", type=float, default=0.05)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--L", type=int, default=2000)
    ap.add_argument("--beta", type=float, default=0.1)
    ap.add_argument("--seed", type=int, default=12345)
    ap.add_argument("--out", required=True)
    ap.add_argument("--log", default=None)
    ap.add_argument("--dilation", choices=("manhattan", "chebyshev"), default="manhattan")
    args = ap.parse_args()
    logf = open(args.log, "w") if args.log else None

    def log(msg):
        print(msg, flush=True)
        if logf:
            logf.write(msg + "\n")
            logf.flush()

    t0 = time.perf_counter()
    net = TileProposer(seed=args.seed)
    data = build_dataset(args.pairs, args.seed, args.L, args.beta, net, log=log)
    nval = max(1, int(len(data) * args.val))
    val, tr = data[:nval], data[nval:]
    hist, pw = train(net, tr, args.L, args.epochs, args.lr, log=log)
    thr, kept = calibrate(net, val, args.L, manhattan=args.dilation == "manhattan")
    net.threshold = thr
    net.manhattan = args.dilation == "manhattan"
    info = {"train_pairs": len(tr), "val_pairs": len(val), "epochs": args.epochs,
            "loss_history": hist, "pos_weight": pw, "threshold": thr,
            "val_kept_fraction": kept, "dilation": args.dilation, "L": args.L,
            "seconds": time.perf_counter() - t0}
    log(json.dumps(info))
    net.save(args.out, info=json.dumps(info))


if __name__ == "__main__":
    main()
