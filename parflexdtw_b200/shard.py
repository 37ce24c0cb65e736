"""Multi-GPU alignment: pairs of a batch, or the tiles of one long pair,
sharded across ranks (one process per GPU, launched by torchrun).

Batches: pairs are independent (one alignment never needs another's data),
so a batch splits with no data-path collective: each rank aligns its share
with ``parflex_batch`` on its own device, and one ``gather_object`` brings
(best cost, path) to rank 0 at the end.  Shares are balanced by DP cells
(N x M), largest pair first, each to the least-loaded rank.

One long pair: stage-1 tiles are independent (Parflex.py:421-454), so each
rank runs the cost and stage 1 of a contiguous range of tile indices
(``shard_tiles``, balanced by cells) under a tile mask, plus the edge-tensor
step of stage 2 for those tiles.  One exchange step follows: rank 0 gathers
every tile's edge costs, start encodings and overlap costs (contiguous
slices of the tile-major edge arrays, a few MB) and reduces the valid masks
with MAX.  Rank 0 runs the propagation, the scan and the tile chain of the
stitched backtrace; it broadcasts the crossed tiles, and their owners send
only those tiles' packed backpointers (``exchange_backptr``) before rank 0
walks the path.  Over NCCL the tensors stay on the device; over gloo they
are staged through host memory.
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


# -- one long pair, tiles sharded ---------------------------------------------

def tile_cells(n1, n2, N, M, Lb, hop):
    """DP cells of every tile in tile order (t = i * n2 + j)."""
    rows = [min(Lb, N - i * hop) for i in range(n1)]
    cols = [min(Lb, M - j * hop) for j in range(n2)]
    return [r * c for r in rows for c in cols]


def shard_tiles(cells, world_size):
    """Contiguous tile-index ranges [lo, hi), one per rank, balanced by cells
    (each boundary at the prefix sum closest to its share).  Rank 0, which
    runs stage 2, always gets a tile; other ranges may be empty when there
    are fewer tiles than ranks."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    pre = np.concatenate([[0], np.cumsum(np.asarray(cells, dtype=np.int64))])
    nt, total = len(cells), int(pre[-1])
    bounds = [0]
    for k in range(1, world_size):
        target = total * k / world_size
        t = int(np.searchsorted(pre, target))
        if t > 0 and (t > nt or target - pre[t - 1] <= pre[t] - target):
            t -= 1
        bounds.append(min(max(t, bounds[-1], 1 if nt else 0), nt))
    bounds.append(nt)
    return [(bounds[r], bounds[r + 1]) for r in range(world_size)]


def _comm_device(group):
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def exchange_edges(edge_D, edge_P, edge_Cf, valid, ranges, group=None):
    """Gather every rank's tile slices of the tile-major edge arrays into
    rank 0's (in place) and reduce the valid masks with MAX there.

    All four arrays hold n1 * n2 * 2 * L entries in tile order; rank r's
    tiles are ``ranges[r]``.  Every rank calls this with its own arrays.
    """
    import torch
    import torch.distributed as dist
    rank, ws = dist.get_rank(group), dist.get_world_size(group)
    dev = _comm_device(group)
    nt = sum(hi - lo for lo, hi in ranges)
    spt = edge_D.numel() // nt if nt else 0
    lens = [(hi - lo) * spt for lo, hi in ranges]
    width = max(max(lens), 1)
    lo = ranges[rank][0] * spt
    n = lens[rank]
    flat = [x.reshape(-1) for x in (edge_D, edge_P, edge_Cf, valid)]
    pk64 = torch.zeros(2, width, dtype=torch.float64, device=dev)
    pk32 = torch.zeros(width, dtype=torch.int32, device=dev)
    pk64[0, :n].copy_(flat[0][lo:lo + n])
    pk64[1, :n].copy_(flat[2][lo:lo + n])
    pk32[:n].copy_(flat[1][lo:lo + n])
    g64 = [torch.empty_like(pk64) for _ in range(ws)] if rank == 0 else None
    g32 = [torch.empty_like(pk32) for _ in range(ws)] if rank == 0 else None
    dist.gather(pk64, g64, dst=0, group=group)
    dist.gather(pk32, g32, dst=0, group=group)
    # a rank without tiles ran nothing: its valid mask contributes no marks
    # (a copy: the collective gets a tensor of its own allocator, not the plan's)
    vm = flat[3].to(dev, copy=True) if n else torch.zeros(flat[3].numel(), dtype=flat[3].dtype,
                                                          device=dev)
    dist.reduce(vm, dst=0, op=dist.ReduceOp.MAX, group=group)
    if rank != 0:
        return
    for r in range(1, ws):
        a, m = ranges[r][0] * spt, lens[r]
        if m == 0:
            continue
        flat[0][a:a + m].copy_(g64[r][0, :m])
        flat[2][a:a + m].copy_(g64[r][1, :m])
        flat[1][a:a + m].copy_(g32[r][:m])
    flat[3].copy_(vm)


def _owner(t, ranges):
    for r, (lo, hi) in enumerate(ranges):
        if lo <= t < hi:
            return r
    raise ValueError(f"tile {t} has no owner")


def exchange_backptr(bw, crossed, ranges, group=None):
    """Bring the packed backpointers of the crossed tiles to rank 0.

    ``bw`` is this rank's (n1 * n2, b_words) backpointer array; ``crossed``
    the crossed tile indices on rank 0 (ignored elsewhere: rank 0 broadcasts
    them, at most 101).  Returns the crossed tile list on every rank.
    """
    import torch
    import torch.distributed as dist
    rank, ws = dist.get_rank(group), dist.get_world_size(group)
    dev = _comm_device(group)
    msg = torch.full((102,), -1, dtype=torch.int64, device=dev)
    if rank == 0:
        c = [int(t) for t in crossed]
        if len(c) > 101:
            raise ValueError("the stitched backtrace crosses at most 101 tiles")
        msg[0] = len(c)
        if c:
            msg[1:1 + len(c)] = torch.tensor(c, dtype=torch.int64)
    dist.broadcast(msg, src=0, group=group)
    n = int(msg[0])
    tiles = [int(t) for t in msg[1:1 + n].tolist()]
    mine = [[t for t in tiles if _owner(t, ranges) == r] for r in range(ws)]
    cnt = max(len(m) for m in mine[1:]) if ws > 1 else 0
    if cnt == 0:
        return tiles
    bwords = bw.shape[1]
    pk = torch.zeros(cnt, bwords, dtype=bw.dtype, device=dev)
    for k, t in enumerate(mine[rank] if rank else []):
        pk[k].copy_(bw[t])
    got = [torch.empty_like(pk) for _ in range(ws)] if rank == 0 else None
    dist.gather(pk, got, dst=0, group=group)
    if rank == 0:
        for r in range(1, ws):
            for k, t in enumerate(mine[r]):
                bw[t].copy_(got[r][k])
    return tiles


class ShardedPair:
    """One long pair with its tiles sharded across the ranks of ``group``
    (default: the default process group), set up once and aligned any
    number of times: per rank a plan that holds the cost slabs of its own
    contiguous tile range only (``shard_tiles``, balanced by cells).

    ``run(beta, F1d, F2d)`` is one alignment: each rank builds the cost of
    its tiles from the device features (when given; else the last loaded
    cost is reused) and runs stage 1 and the edge step of stage 2 on them;
    rank 0 gathers the edges, runs the rest of stage 2 and the tile chain,
    the owners of the crossed tiles send their backpointers, and rank 0
    walks the path.  Rank 0 returns ``(best_cost, wp)``, the others None.
    Every rank takes the same collective steps in the same order, failures
    included (a stage-1 failure anywhere ends the call on every rank).
    """

    def __init__(self, N, M, steps, weights, L=None, group=None, precision="fp64"):
        import torch.distributed as dist
        from .parflex import DEFAULT_CHUNK_LENGTH
        from .plan import Plan
        self.group = group
        self.ws = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.L = int(DEFAULT_CHUNK_LENGTH if L is None else L)
        self.plan = Plan(int(N), int(M), self.L, steps, weights, precision=precision)
        p = self.plan
        self.cells = tile_cells(p.n1, p.n2, p.N, p.M, self.L, p.hop)
        self.ranges = shard_tiles(self.cells, self.ws)
        self.lo, self.hi = self.ranges[self.rank]
        if self.hi > self.lo:
            p.set_tile_range(self.lo, self.hi)  # cost slabs of the own tiles only

    @property
    def own_cells(self):
        return int(sum(self.cells[self.lo:self.hi]))

    def edge_exchange_bytes(self):
        """Bytes rank 0 receives in the edge exchange per alignment: 20 B
        per edge slot (D f64, overlap cost f64, start i32) of the other
        ranks' tiles, plus the valid mask reduction (1 B per slot per rank)."""
        if self.ws == 1:
            return 0
        spt = 2 * self.L
        other = sum(hi - lo for r, (lo, hi) in enumerate(self.ranges) if r)
        return other * spt * 20 + (self.ws - 1) * len(self.cells) * spt

    def run(self, beta, F1d=None, F2d=None, events=False):
        """One alignment (see the class docstring).  ``events``: record CUDA
        events around this rank's cost build and stage 1, read back with
        ``local_ms()``."""
        import torch
        import torch.distributed as dist
        plan, ws, rank, group = self.plan, self.ws, self.rank, self.group
        failure = None
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)] if events else None
        try:
            if self.hi > self.lo:
                if ev:
                    ev[0].record()
                if F1d is not None:
                    plan.load_features(F1d, F2d)
                if ev:
                    ev[1].record()
                plan.stage1()
                if ev:
                    ev[2].record()
                plan.edges()
                plan.result(raise_no_endpoint=False)  # synchronises; raises if a wait ran out
            self._ev = ev if self.hi > self.lo else None
        except Exception as e:  # noqa: BLE001 - re-raised below, after the reduction
            failure = e
        status = 0 if failure is None else 1
        if ws > 1:
            st = torch.tensor([status], dtype=torch.int32, device=_comm_device(group))
            dist.all_reduce(st, op=dist.ReduceOp.MAX, group=group)
            status = int(st.item())
        if failure is not None:
            raise failure
        if status:
            raise RuntimeError("stage 1 of a tile shard failed on another rank")
        if ws > 1:
            exchange_edges(plan.view("EDGE_D"), plan.view("EDGE_P"), plan.view("EDGE_CF"),
                           plan.view("VALID"), self.ranges, group)
        crossed = []
        if rank == 0:
            # the rest of stage 2 reads no cost: the tile range may stay
            plan.prop()
            plan.scan(beta)
            crossed = [int(i) * plan.n2 + int(j) for i, j in plan.chain()]
        if ws > 1:
            bw = plan.view("BACKPTR").view(torch.int32).reshape(plan.n1 * plan.n2, -1)
            exchange_backptr(bw, crossed, self.ranges, group)
        if rank != 0:
            torch.cuda.synchronize()
            return None
        plan.stitch()
        best, end, found, n = plan.result()
        wp = plan.path(n)
        if wp.shape[0] == 0:
            return best, np.array([[], []], dtype=np.int64)
        return best, np.ascontiguousarray(wp.T)

    def local_ms(self):
        """(cost build ms, stage-1 ms) of this rank's last ``run(events=True)``
        ((0, 0) for a rank without tiles)."""
        ev = getattr(self, "_ev", None)
        if not ev:
            return 0.0, 0.0
        return ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])

    def close(self):
        self.plan.close()


def parflex_sharded(F1, F2, steps, weights, beta, L=None, group=None, precision="fp64"):
    """ParFlex of one long pair with its tiles sharded across the ranks of
    ``group`` (default: the default process group).

    Every rank passes the same features (d x N and d x M, FP64); rank 0
    returns ``(best_cost, wp)`` exactly as ``parflex`` on the same cost
    would (``precision="fp32"``: as a single FP32-form plan would), the
    other ranks None.  Each rank builds the cost and runs stage 1 only for
    its own tiles; see the module docstring for the exchange.
    """
    from .parflex import _features_to_device
    F1d, F2d = _features_to_device(F1), _features_to_device(F2)
    sp = ShardedPair(F1d.shape[1], F2d.shape[1], steps, weights, L=L, group=group,
                     precision=precision)
    try:
        return sp.run(beta, F1d, F2d)
    finally:
        sp.close()
