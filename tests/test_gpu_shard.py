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
from parflexdtw_b200.plan import Plan  # noqa: E402
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


def _rank_main(rank, port, world, seed, n, m, Lb, q, wts=WTS):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ.setdefault("GLOO_SOCKET_IFNAME", "lo")
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        F1, F2 = _pair(seed, n, m)
        res = parflex_sharded(F1, F2, STD, wts, 0.1, L=Lb)
        q.put((rank, None if res is None else (float(res[0]), res[1].tolist())))
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, repr(e)))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,seed,n,m,Lb,wts", [(2, 11, 1500, 1800, 400, WTS),
                                                   (3, 12, 2300, 1900, 500, WTS),
                                                   (2, 13, 300, 350, 400, WTS),
                                                   (2, 16, 1700, 1400, 300, [1.25, 3.0, 3.0])])
def test_tile_sharded_pair_vs_oracle(oracle_mod, world, seed, n, m, Lb, wts):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, port, world, seed, n, m, Lb, q, wts))
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
    ref = oracle_mod.parflex_full(C, STD, wts, 0.1, Lb)
    assert best == ref["best_cost"]
    assert np.array_equal(wp, ref["wp"])
    b1, wp1 = pf.parflex(C, STD, wts, 0.1, L=Lb, profile_dir=None)
    assert b1 == best and np.array_equal(wp1, wp)


def _rank_main_fp32(rank, port, world, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ.setdefault("GLOO_SOCKET_IFNAME", "lo")
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(17)
        F1, F2 = W.warped_pair(rng, 1600, 1500, d=64, noise=0.1, latent="gaussian")
        res = parflex_sharded(F1, F2, STD, WTS, 0.1, L=400, precision="fp32")
        q.put((rank, None if res is None else (float(res[0]), res[1].tolist())))
    except Exception as e:  # report instead of hanging the parent
        q.put((rank, repr(e)))
        raise
    finally:
        dist.destroy_process_group()


def test_tile_sharded_fp32_form_vs_single_plan():
    """The FP32 form sharded over two ranks equals one FP32-form plan."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main_fp32, args=(r, port, 2, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=600) for _ in procs)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0, got
    assert got[1] is None
    rng = np.random.default_rng(17)
    F1, F2 = W.warped_pair(rng, 1600, 1500, d=64, noise=0.1, latent="gaussian")
    p = Plan(F1.shape[1], F2.shape[1], 400, STD, WTS, precision="fp32")
    p.load_features(torch.from_numpy(np.ascontiguousarray(F1)).cuda(),
                    torch.from_numpy(np.ascontiguousarray(F2)).cuda())
    p.run(None, 0.1)
    best, _, _, n = p.result()
    wp = p.path(n).T
    assert got[0][0] == best
    assert np.array_equal(np.asarray(got[0][1], dtype=np.int64), wp)
    p.close()


def test_tile_sharded_single_process_vs_oracle(oracle_mod):
    """Without a process group the whole pair is rank 0's shard."""
    F1, F2 = _pair(14, 1200, 1000)
    best, wp = parflex_sharded(F1, F2, STD, WTS, 0.1, L=300)
    ref = oracle_mod.parflex_full(W.cost_matrix_det(F1, F2), STD, WTS, 0.1, 300)
    assert best == ref["best_cost"] and np.array_equal(wp, ref["wp"])


def _written_bp_words(plan, t):
    """Indices of tile t's packed backpointer words that stage 1 writes: per
    strip k, 16-step block p and lane, the (A, B) word pair of rows
    64k + 2 lane (+1), for lanes whose first row is inside the tile."""
    i, j = divmod(t, plan.n2)
    R = min(plan.L, plan.N - i * plan.hop)
    W_ = min(plan.L, plan.M - j * plan.hop)
    nS = -(-R // 64)
    nP = -(-(W_ + 63) // 16)
    k, p, lane = np.meshgrid(np.arange(nS), np.arange(nP), np.arange(32), indexing="ij")
    keep = 64 * k + 2 * lane < R
    base = 2 * ((k * nP + p) * 32 + lane)[keep]
    return np.sort(np.concatenate([base, base + 1]))


def test_tile_range_plan_holds_its_tiles_only():
    """A ranged plan: packed slabs for its tiles, stage 1 on them alone with
    the same edges and backpointers as the full plan, and a mask that stays."""
    F1, F2 = _pair(15, 1300, 1500)
    F1d, F2d = (torch.from_numpy(np.ascontiguousarray(F)).cuda() for F in (F1, F2))
    full = Plan(F1.shape[1], F2.shape[1], 400, STD, WTS)
    full.load_features(F1d, F2d)
    full.stage1()
    nt = full.n1 * full.n2
    lo, hi = 3, nt - 2
    part = Plan(F1.shape[1], F2.shape[1], 400, STD, WTS)
    part.set_tile_range(lo, hi)
    with pytest.raises(ValueError):
        part.set_tile_range(0, 1)
    with pytest.raises(ValueError):
        part.set_tile_mask(None)
    part.load_features(F1d, F2d)
    part.stage1()
    torch.cuda.synchronize()
    assert part.view("COST").numel() == full.view("COST").numel() // nt * (hi - lo)
    eD, fD = part.host("EDGE_D").reshape(nt, -1), full.host("EDGE_D").reshape(nt, -1)
    eP, fP = part.host("EDGE_P").reshape(nt, -1), full.host("EDGE_P").reshape(nt, -1)
    assert np.array_equal(eD[lo:hi], fD[lo:hi]) and np.array_equal(eP[lo:hi], fP[lo:hi])
    assert np.all(np.isinf(eD[:lo])) and np.all(eP[hi:] == 0)
    bw_p = part.host("BACKPTR").reshape(nt, -1)
    bw_f = full.host("BACKPTR").reshape(nt, -1)
    for t in range(lo, hi):  # the words stage 1 writes (the rest is never read)
        w = _written_bp_words(part, t)
        assert np.array_equal(bw_p[t][w], bw_f[t][w]), t
    with pytest.raises(ValueError):
        Plan(100, 100, 50, STD, WTS).set_tile_range(2, 2)
    part.close()
    full.close()
