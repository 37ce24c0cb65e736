"""Multi-rank batches on CPU: two gloo ranks shard a batch of pairs and rank 0
gathers the results.  The aligner here is the oracle (no GPU): the test
checks the partition, the balancing and that the gathered results equal a
single-process run, in input order."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from parflexdtw_b200 import workloads as W  # noqa: E402
from parflexdtw_b200.shard import (exchange_backptr, exchange_edges,  # noqa: E402
                                   parflex_batch_sharded, shard_pairs, shard_tiles,
                                   tile_cells)

STD = [(1, 1), (1, 2), (2, 1)]
WTS = [2.0, 3.0, 3.0]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _pairs():
    rng = np.random.default_rng(42)
    return [W.warped_pair(rng, n, m, pad_frac=0.1)
            for n, m in [(300, 350), (120, 160), (500, 420), (260, 300), (90, 100)]]


def _oracle_aligner(pairs, steps, weights, beta, L=None):
    from oracle import build_oracle, oracle
    build_oracle.build()
    out = []
    for k, (F1, F2) in enumerate(pairs):
        Lb = L[k] if np.ndim(L) else L
        best, wp = oracle.parflex(W.cost_matrix_det(F1, F2), steps, weights, beta, Lb)
        out.append((best, wp))
    return out


def _rank_main(rank, port, world, Ls, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = parflex_batch_sharded(_pairs(), STD, WTS, 0.1, L=Ls, aligner=_oracle_aligner)
        if rank == 0:
            q.put([(float(b), wp.tolist()) for b, wp in res])
        else:
            q.put(res is None)
    finally:
        dist.destroy_process_group()


def test_shard_partition_and_balance():
    shapes = [(1000, 1200), (50, 60), (900, 800), (400, 400), (1000, 1000), (10, 10)]
    for ws in (1, 2, 3, 8):
        parts = shard_pairs(shapes, ws)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(shapes)))
        loads = [sum(shapes[i][0] * shapes[i][1] for i in p) for p in parts]
        biggest = max(n * m for n, m in shapes)
        assert max(loads) - min(loads) <= biggest
    with pytest.raises(ValueError):
        shard_pairs(shapes, 0)


@pytest.mark.parametrize("Ls", [64, [64, 32, 100, 50, 17]])
def test_two_gloo_ranks_gather_in_order(Ls):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, 2, Ls, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    gathered = next(g for g in got if isinstance(g, list))
    assert any(g is True for g in got)  # rank 1 returned None
    single = _oracle_aligner(_pairs(), STD, WTS, 0.1, L=Ls)
    assert len(gathered) == len(single)
    for (b, wp), (b1, wp1) in zip(gathered, single):
        assert b == b1 and np.array_equal(np.asarray(wp), wp1)


# -- one long pair, tiles sharded: the host-side exchange on gloo ranks ------

NT, SPT, BW = 7, 10, 6  # tiles, edge slots per tile (2 * L), backpointer words per tile


def _truth():
    rng = np.random.default_rng(5)
    D = rng.standard_normal(NT * SPT)
    D[::7] = np.inf
    P = rng.integers(-50, 50, NT * SPT).astype(np.int32)
    Cf = rng.random(NT * SPT)
    bw = rng.integers(-2**31, 2**31 - 1, (NT, BW)).astype(np.int32)
    return D, P, Cf, bw


def _exchange_main(rank, port, world, ranges, crossed, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        D, P, Cf, bw = _truth()
        lo, hi = ranges[rank]
        own = np.zeros(NT * SPT, bool)
        own[lo * SPT:hi * SPT] = True
        # what a masked stage 1 leaves outside the rank's tiles: +inf, 0 and
        # garbage; valid marks differ per rank
        tD = torch.from_numpy(np.where(own, D, np.inf))
        tP = torch.from_numpy(np.where(own, P, 0).astype(np.int32))
        tCf = torch.from_numpy(np.where(own, Cf, -7.0 - rank))
        valid = np.random.default_rng(100 + rank).integers(0, 2, NT * SPT).astype(np.uint8)
        tV = torch.from_numpy(valid.copy())
        exchange_edges(tD, tP, tCf, tV, ranges)
        tbw = torch.from_numpy(bw.copy())
        for t in range(NT):
            if not lo <= t < hi:
                tbw[t] = 1000 + rank
        tiles = exchange_backptr(tbw, crossed if rank == 0 else None, ranges)
        q.put((rank, tD.numpy(), tP.numpy(), tCf.numpy(), tV.numpy(), tbw.numpy(), tiles))
    finally:
        dist.destroy_process_group()


def test_shard_tiles_partition():
    cells = tile_cells(4, 5, 1700, 2100, 500, 400)
    assert len(cells) == 20 and cells[0] == 500 * 500 and cells[-1] == (1700 - 1200) * (2100 - 1600)
    for ws in (1, 2, 3, 8, 25):
        rg = shard_tiles(cells, ws)
        assert rg[0][0] == 0 and rg[-1][1] == 20 and rg[0][1] >= 1
        assert all(a[1] == b[0] and a[0] <= a[1] for a, b in zip(rg, rg[1:]))
        loads = [sum(cells[lo:hi]) for lo, hi in rg]
        if ws <= 3:
            assert max(loads) - sum(cells) / ws <= max(cells)
    assert shard_tiles([9], 3) == [(0, 1), (1, 1), (1, 1)]
    with pytest.raises(ValueError):
        shard_tiles(cells, 0)


def test_shard_tiles_random_properties():
    """Random tile sizes and rank counts: contiguous cover in order, rank 0
    never empty, every share within one tile of the even split."""
    rng = np.random.default_rng(8)
    for _ in range(300):
        nt = int(rng.integers(1, 60))
        ws = int(rng.integers(1, 12))
        cells = rng.integers(1, 10_000, nt).tolist()
        rg = shard_tiles(cells, ws)
        assert len(rg) == ws and rg[0][0] == 0 and rg[-1][1] == nt and rg[0][1] >= 1
        assert all(a[1] == b[0] and a[0] <= a[1] for a, b in zip(rg, rg[1:]))
        pre = np.concatenate([[0], np.cumsum(cells)])
        for r in range(1, ws):  # each boundary within one tile of its share
            b = rg[r][0]
            target = pre[-1] * r / ws
            lo = pre[b - 1] if b > 0 else 0
            hi = pre[b + 1] if b < nt else pre[-1]
            assert lo <= target <= hi or b == rg[r - 1][0] or b == 1


@pytest.mark.parametrize("world,ranges", [(2, [(0, 3), (3, 7)]),
                                          (3, [(0, 2), (2, 2), (2, 7)])])
def test_exchange_edges_and_backptr_gloo(world, ranges):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    crossed = [6, 4, 3, 1, 0]
    procs = [ctx.Process(target=_exchange_main, args=(r, port, world, ranges, crossed, q))
             for r in range(world)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        r, *rest = q.get(timeout=300)
        got[r] = rest
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    D, P, Cf, bw = _truth()
    tD, tP, tCf, tV, tbw, tiles = got[0]
    assert np.array_equal(tD, D) and np.array_equal(tP, P) and np.array_equal(tCf, Cf)
    want_v = np.zeros(NT * SPT, np.uint8)
    for r in range(world):
        if ranges[r][1] > ranges[r][0]:  # a rank without tiles contributes no marks
            want_v |= np.random.default_rng(100 + r).integers(0, 2, NT * SPT).astype(np.uint8)
    assert np.array_equal(tV, want_v)
    for t in crossed:
        assert np.array_equal(tbw[t], bw[t]), t
    for r in range(world):
        assert got[r][-1] == crossed


# -- failure on one rank: every rank leaves the call, none waits forever ------

class _FakePlan:
    """Host stand-in for Plan: stage 1 fails on the rank named by FAIL_RANK."""

    def __init__(self, N, M, Lb, steps, weights, precision="fp64"):
        self.N, self.M, self.L = N, M, Lb
        self.hop = Lb - 1
        self.n1 = max(1, -(-(N - 1) // (Lb - 1)))
        self.n2 = max(1, -(-(M - 1) // (Lb - 1)))
        self.closed = False

    def set_tile_range(self, lo, hi):
        pass

    def load_features(self, F1, F2):
        pass

    def stage1(self):
        if dist.get_rank() == int(os.environ["FAIL_RANK"]):
            raise RuntimeError("a bounded device wait ran out (host fake)")

    def edges(self):
        pass

    def result(self, raise_no_endpoint=True):
        return 0.0, (0,) * 6, False, 0

    def close(self):
        self.closed = True


def _fail_main(rank, port, world, fail_rank, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["FAIL_RANK"] = str(fail_rank)
    import sys

    from parflexdtw_b200.shard import parflex_sharded
    # the package exports a function named parflex: take the modules themselves
    sys.modules["parflexdtw_b200.plan"].Plan = _FakePlan
    sys.modules["parflexdtw_b200.parflex"]._features_to_device = \
        lambda F: torch.as_tensor(np.asarray(F))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        F1 = np.ones((12, 900))
        F2 = np.ones((12, 1000))
        try:
            parflex_sharded(F1, F2, STD, WTS, 0.1, L=300)
            q.put((rank, "returned"))
        except RuntimeError as e:
            q.put((rank, str(e)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("fail_rank", [0, 1])
def test_tile_shard_failure_on_one_rank_ends_all(fail_rank):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fail_main, args=(r, port, 2, fail_rank, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert "bounded device wait" in got[fail_rank]
    assert "another rank" in got[1 - fail_rank]
