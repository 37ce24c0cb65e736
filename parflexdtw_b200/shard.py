"""Multi-GPU batches: pairs sharded across ranks, results gathered on rank 0.

Pairs are independent (one alignment never needs another's data), so a
batch splits across processes — one per GPU, launched by torchrun — with no
data-path collective: each rank aligns its share with ``parflex_batch`` on
its own device, and one ``gather_object`` brings (best cost, path) to rank 0
at the end.  Shares are balanced by DP cells (N x M), largest pair first,
each to the least-loaded rank.
"""
from __future__ import annotations

import numpy as np


def shard_pairs(shapes, world_size):
    """Indices of the pairs each rank aligns (a partition of range(n))."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    cells = [int(n) * int(m) for n, m in shapes]
    order = sorted(range(len(shapes)), key=lambda i: (-cells[i], i))
    load = [0] * world_size
    out = [[] for _ in range(world_size)]
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += cells[i]
    return [sorted(s) for s in out]


def parflex_batch_sharded(pairs, steps, weights, beta, L=None, aligner=None, group=None,
                          **kwargs):
    """``parflex_batch`` over all ranks of the default process group.

    Every rank passes the same ``pairs``; rank 0 returns the list of all
    results (in input order), the other ranks None.  ``aligner`` (default
    ``parflex_batch``) aligns one rank's share; ``L`` may be per pair.
    """
    import torch.distributed as dist
    if aligner is None:
        from .batch import parflex_batch as aligner
    ws = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    shapes = [(np.shape(F1)[1], np.shape(F2)[1]) for F1, F2 in pairs]
    mine = shard_pairs(shapes, ws)[rank]
    Ls = L if (L is None or np.ndim(L) == 0) else [L[i] for i in mine]
    local = aligner([pairs[i] for i in mine], steps, weights, beta, L=Ls, **kwargs) if mine \
        else []
    payload = list(zip(mine, local))
    if ws == 1:
        gathered = [payload]
    else:
        gathered = [None] * ws if rank == 0 else None
        dist.gather_object(payload, gathered, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * len(pairs)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out
