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
from parflexdtw_b200.shard import parflex_batch_sharded, shard_pairs  # noqa: E402

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
