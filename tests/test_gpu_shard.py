"""One long pair with its tiles sharded across ranks (``parflex_sharded``):
two and three gloo ranks, each a process on the same GPU (their kernels never
wait on one another; the exchange goes through host memory), must give
exactly the oracle's and the single-plan best cost and path."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

import parflexdtw_b200 as pf  # noqa: E402
from parflexdtw_b200 import workloads as W  # noqa: E402
from parflexdtw_b200.shard import parflex_sharded  # noqa: E402

STD = [(1, 1), (1, 2), (2, 1)]
WTS = [2.0, 3.0, 3.0]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _pair(seed, n, m):
    return W.warped_pair(np.random.default_rng(seed), n, m, pad_frac=0.1)


def _rank_main(rank, port, world, seed, n, m, Lb, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ.setdefault("GLOO_SOCKET_IFNAME", "lo")
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        F1, F2 = _pair(seed, n, m)
        res = parflex_sharded(F1, F2, STD, WTS, 0.1, L=Lb)
        q.put((rank, None if res is None else (float(res[0]), res[1].tolist())))
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, repr(e)))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,seed,n,m,Lb", [(2, 11, 1500, 1800, 400),
                                               (3, 12, 2300, 1900, 500),
                                               (2, 13, 300, 350, 400)])
def test_tile_sharded_pair_vs_oracle(oracle_mod, world, seed, n, m, Lb):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, world, seed, n, m, Lb, q))
             for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0, got
    assert all(got[r] is None for r in range(1, world)), got
    best, wp = got[0][0], np.asarray(got[0][1], dtype=np.int64)
    F1, F2 = _pair(seed, n, m)
    C = W.cost_matrix_det(F1, F2)
    ref = oracle_mod.parflex_full(C, STD, WTS, 0.1, Lb)
    assert best == ref["best_cost"]
    assert np.array_equal(wp, ref["wp"])
    b1, wp1 = pf.parflex(C, STD, WTS, 0.1, L=Lb, profile_dir=None)
    assert b1 == best and np.array_equal(wp1, wp)


def test_tile_sharded_single_process_vs_oracle(oracle_mod):
    """Without a process group the whole pair is rank 0's shard."""
    F1, F2 = _pair(14, 1200, 1000)
    best, wp = parflex_sharded(F1, F2, STD, WTS, 0.1, L=300)
    ref = oracle_mod.parflex_full(W.cost_matrix_det(F1, F2), STD, WTS, 0.1, 300)
    assert best == ref["best_cost"] and np.array_equal(wp, ref["wp"])
