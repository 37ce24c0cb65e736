"""Batched alignment (pfx_batch_* / parflex_batch) vs the C oracle.

Every pair of a batch must give exactly what the single-pair path and the
oracle give for it (bit-exact best cost, endpoint and path), whatever the
wave packing, the warps per tile, graph replay or direct launch.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import parflexdtw_b200 as pf  # noqa: E402
from parflexdtw_b200 import workloads as W  # noqa: E402
from parflexdtw_b200.autotune import Autotuner  # noqa: E402
from parflexdtw_b200.batch import Batch  # noqa: E402

STD = [(1, 1), (1, 2), (2, 1)]
WTS = [2.0, 3.0, 3.0]


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


def _pairs(seed, sizes, pad=0.1):
    rng = np.random.default_rng(seed)
    return [W.warped_pair(rng, n, m, pad_frac=pad) for n, m in sizes]


SIZES = [(700, 900), (1500, 1200), (333, 410), (1200, 1700), (90, 120), (2100, 2000)]
LS = [128, 300, 64, 500, 17, 256]


@pytest.fixture(scope="module")
def reference(oracle_mod):
    pairs = _pairs(1, SIZES)
    refs = [oracle_mod.parflex_full(W.cost_matrix_det(F1, F2), STD, WTS, 0.1, Lb)
            for (F1, F2), Lb in zip(pairs, LS)]
    return pairs, refs


def _check(b, refs):
    best, end, lens = b.results()
    paths = b.paths(lens)
    for i, ref in enumerate(refs):
        assert best[i] == ref["best_cost"], i
        assert tuple(end[i, :6]) == tuple(ref["best_end"]), i
        assert end[i, 6] == 1
        assert same(paths[i].T, ref["wp"]), i


@pytest.mark.parametrize("cost", ["tile", "slabs"])
@pytest.mark.parametrize("warps", [4, 8, 16])
def test_batch_one_wave_vs_oracle(reference, warps, cost):
    """Either way of building the cost: inside the stage-1 kernel, tile by
    tile ("tile"), or with separate cost kernels ("slabs")."""
    pairs, refs = reference
    b = Batch([(p[0].shape[1], p[1].shape[1]) for p in pairs], LS, STD, WTS, 12, warps=warps,
              cost=cost)
    assert b.waves == 1 and b.warps == warps
    assert b.cost_in_kernel == (cost == "tile")
    b.load(pairs)
    b.run(0.1)
    _check(b, refs)
    # graph replay on fresh features gives the same answers again
    b.run(0.1)
    _check(b, refs)
    b.close()


@pytest.mark.parametrize("cost", ["tile", "slabs"])
def test_batch_waves_and_direct_launch(reference, cost):
    """A small slab pool splits a batch with separate cost kernels into
    waves; with the cost built inside stage 1 every pair runs in one wave
    whatever the pool would have held."""
    pairs, refs = reference
    shapes = [(p[0].shape[1], p[1].shape[1]) for p in pairs]
    b = Batch(shapes, LS, STD, WTS, 12, wave_bytes=56 << 20, warps=4, cost=cost)
    if cost == "slabs":
        assert b.waves >= 2
    else:
        assert b.waves == 1 and b.cost_in_kernel
    b.load(pairs)
    b.run(0.1, use_graph=False)
    _check(b, refs)
    b.run(0.1, use_graph=True)
    _check(b, refs)
    b.close()


@pytest.mark.parametrize("d,steps,weights", [
    (1, STD, WTS),
    (5, [(1, 1), (2, 1)], [1.0, 2.5]),
    (16, [(1, 2), (1, 1), (2, 1)], [3.0, 1.25, 3.0]),
    (13, [(1, 1)], [2.0]),
])
def test_batch_cost_in_kernel_dims_and_steps_vs_oracle(oracle_mod, d, steps, weights):
    """The in-kernel cost for every feature dimension it takes (both of its
    unrolled forms, d <= 12 and 13..16) and other step sets, uneven tile
    lengths and tiles of one row or column: bit-exact with the oracle on the
    fixed-order host cost, and with the batch that builds slabs first."""
    sizes = [(700, 900), (301, 64), (65, 640), (1200, 1100)]
    Ls = [256, 64, 128, 500]
    rng = np.random.default_rng(31 + d)
    pairs = [W.warped_pair(rng, n, m, d=d, noise=0.1, latent="gaussian") if d > 1 else
             (np.abs(rng.standard_normal((1, n))) + 0.1, np.abs(rng.standard_normal((1, m))) + 0.1)
             for n, m in sizes]
    shapes = [(p[0].shape[1], p[1].shape[1]) for p in pairs]
    refs = [oracle_mod.parflex_full(W.cost_matrix_det(F1, F2), steps, weights, 0.1, Lb)
            for (F1, F2), Lb in zip(pairs, Ls)]
    got = {}
    for cost in ("tile", "slabs"):
        b = Batch(shapes, Ls, steps, weights, d, cost=cost)
        assert b.cost_in_kernel == (cost == "tile")
        b.load(pairs)
        b.run(0.1)
        _check(b, refs)
        got[cost] = [b.plan(i).host("D_ARR") for i in range(b.n)]
        b.close()
    for x, y in zip(got["tile"], got["slabs"]):
        assert same(x, y)


@pytest.mark.parametrize("d,steps,weights", [
    (12, STD, WTS),
    (5, [(1, 1), (2, 1)], [1.0, 2.5]),
    (40, STD, WTS),
])
def test_batch_cost_fma_vs_oracle(oracle_mod, d, steps, weights):
    """PFX_BATCH_COST_FMA: the cost as a fixed-order FMA chain, bit-exact with
    the oracle's fma chain (oracle_cost_fma), and the whole alignment
    bit-exact with the oracle on that cost; both cost kernels (d <= 16 and the
    chunked d > 16 one), masked runs and completions included."""
    sizes = [(700, 900), (1500, 1200), (333, 410), (1200, 1700)]
    Ls = [256, 300, 128, 500]
    rng = np.random.default_rng(41 + d)
    pairs = [W.warped_pair(rng, n, m, d=d, noise=0.1, latent="gaussian") for n, m in sizes]
    shapes = [(p[0].shape[1], p[1].shape[1]) for p in pairs]
    Cs = [oracle_mod.cost_matrix_fma(F1, F2) for F1, F2 in pairs]
    refs = [oracle_mod.parflex_full(C, steps, weights, 0.1, Lb) for C, Lb in zip(Cs, Ls)]
    b = Batch(shapes, Ls, steps, weights, d, cost_fma=True)
    assert b.cost_fma
    b.load(pairs)
    b.run(0.1)
    _check(b, refs)
    torch.cuda.synchronize()
    assert same(b.plan(3).cost_matrix(), Cs[3])
    # masked run on every tile, then completion of one pair from a sparse mask
    grids = [(-(-(n - 1) // (Lb - 1)), -(-(m - 1) // (Lb - 1))) for (n, m), Lb in zip(shapes, Ls)]
    b.set_masks(torch.ones(sum(a * c for a, c in grids), dtype=torch.uint8, device="cuda"))
    b.run(0.1, use_graph=False)
    _check(b, refs)
    rng2 = np.random.default_rng(3)
    sparse = torch.from_numpy((rng2.random(sum(a * c for a, c in grids)) < 0.5)
                              .astype(np.uint8)).cuda()
    b.set_masks(sparse)
    b.run(0.1, use_graph=False)
    for i, r in enumerate(refs):
        bc, wp = b.complete(i, 0.1)
        assert bc == r["best_cost"] and same(wp.T, r["wp"]), i
    b.close()
    with pytest.raises(ValueError):
        Batch(shapes, Ls, steps, weights, d, cost_fma=True, cost="tile")


def test_batch_beta_change_rerecords(oracle_mod):
    pairs = _pairs(2, [(800, 950), (640, 600)])
    C = [W.cost_matrix_det(F1, F2) for F1, F2 in pairs]
    b = Batch([(p[0].shape[1], p[1].shape[1]) for p in pairs], 200, STD, WTS, 12)
    b.load(pairs)
    for beta in (0.1, 0.3, 0.1):
        b.run(beta)
        best, end, lens = b.results()
        paths = b.paths(lens)
        for i in range(2):
            ref = oracle_mod.parflex_full(C[i], STD, WTS, beta, 200)
            assert best[i] == ref["best_cost"]
            assert same(paths[i].T, ref["wp"])
    b.close()


def test_batch_plan_views_match_single_pair(reference, oracle_mod):
    """Stage-2 intermediates of a pair inside a batch equal the oracle's."""
    pairs, refs = reference
    b = Batch([(p[0].shape[1], p[1].shape[1]) for p in pairs], LS, STD, WTS, 12)
    b.load(pairs)
    b.run(0.1)
    torch.cuda.synchronize()
    for i in (0, 3):
        p = b.plan(i)
        assert same(p.host("D_ARR"), refs[i]["D_arr"])
        assert same(p.host("L_ARR"), refs[i]["L_arr"])
        bc, be, found, n = p.result()
        assert bc == refs[i]["best_cost"] and found
    b.close()


def test_parflex_batch_api_matches_parflex(reference):
    pairs, refs = reference
    out = pf.parflex_batch(pairs, STD, WTS, 0.1, L=LS)
    for (best, wp), ref, (F1, F2), Lb in zip(out, refs, pairs, LS):
        assert best == ref["best_cost"]
        assert same(wp, ref["wp"])
        b1, wp1 = pf.parflex(W.cost_matrix_det(F1, F2), STD, WTS, 0.1, L=Lb, profile_dir=None)
        assert b1 == best and same(wp1, wp)


def test_autotuner_picks_candidates_and_stays_exact(oracle_mod):
    sizes = [(900, 1000), (1000, 1300), (5000, 4500), (4200, 5200)]
    pairs = _pairs(3, sizes)
    t = Autotuner(candidates_L=(250, 500), candidates_warps=(4, 16), probe_pairs=2,
                  bucket_edges=(3000,), repeats=1)
    Ls, warps = t.choose([(p[0].shape[1], p[1].shape[1]) for p in pairs], STD, WTS, 12)
    assert set(Ls) <= {250, 500} and warps in (4, 16)
    assert Ls[0] == Ls[1] and Ls[2] == Ls[3]  # one choice per bucket
    assert len(t.log) == 8  # 2 buckets x 2 L x 2 warps probes
    out = pf.parflex_batch(pairs, STD, WTS, 0.1, tuner=t)
    for (best, wp), (F1, F2), Lb in zip(out, pairs, Ls):
        ref = oracle_mod.parflex_full(W.cost_matrix_det(F1, F2), STD, WTS, 0.1, Lb)
        assert best == ref["best_cost"]
        assert same(wp, ref["wp"])


def test_batch_fp64_wide_features_vs_oracle(oracle_mod):
    """d > 16: the FP64 cost sums the features 16 at a time, same order."""
    sizes = [(500, 640), (800, 700), (300, 350)]
    rng = np.random.default_rng(9)
    pairs = [W.warped_pair(rng, n, m, d=40, noise=0.1, latent="gaussian") for n, m in sizes]
    b = Batch([(p[0].shape[1], p[1].shape[1]) for p in pairs], 200, STD, WTS, 40)
    b.load(pairs)
    b.run(0.1)
    refs = [oracle_mod.parflex_full(W.cost_matrix_det(F1, F2), STD, WTS, 0.1, 200)
            for F1, F2 in pairs]
    _check(b, refs)
    assert same(b.plan(1).cost_matrix(), W.cost_matrix_det(*pairs[1]))
    b.close()


def test_batch_fp32_vs_oracle(oracle_mod):
    """FP32 form batch: per pair, the oracle's FP32 form on the device's own
    tensor-core cost; also equal to the single-pair FP32 plan."""
    sizes = [(900, 1100), (1500, 1300), (400, 380), (2200, 2000)]
    rng = np.random.default_rng(10)
    pairs = [W.warped_pair(rng, n, m, d=128, noise=0.1, latent="gaussian") for n, m in sizes]
    shapes = [(p[0].shape[1], p[1].shape[1]) for p in pairs]
    b = Batch(shapes, [300, 500, 128, 1000], STD, WTS, 128, precision="fp32", warps=8)
    b.load(pairs)
    b.run(0.1)
    torch.cuda.synchronize()
    refs = [oracle_mod.parflex_full(b.plan(i).cost_matrix().astype(np.float64), STD, WTS, 0.1,
                                    b.L[i], fp32=True) for i in range(b.n)]
    _check(b, refs)
    p = pf.Plan(shapes[3][0], shapes[3][1], 1000, STD, WTS, precision="fp32")
    p.load_features(torch.from_numpy(pairs[3][0]).cuda(), torch.from_numpy(pairs[3][1]).cuda())
    p.run(None, 0.1)
    best, end, found, n = p.result()
    assert best == refs[3]["best_cost"]
    b.close()


def test_batch_fp32_masked_vs_unmasked(oracle_mod):
    """Masked FP32 batches: all-ones masks and path-dilated masks give the
    unmasked FP32 results bit for bit, which equal the oracle's FP32 form on
    the device's own cost; so does PrunedBatch in the FP32 form."""
    from parflexdtw_b200.prune import tiles_on_path
    sizes = [(1900, 2100), (2600, 2300), (900, 1000), (1500, 1700)]
    rng = np.random.default_rng(21)
    pairs = [W.warped_pair(rng, n, m, d=12, noise=0.1, latent="gaussian") for n, m in sizes]
    shapes = [(p[0].shape[1], p[1].shape[1]) for p in pairs]
    L = 300
    b = Batch(shapes, L, STD, WTS, 12, precision="fp32", warps=4)
    b.load(pairs)
    b.run(0.1, use_graph=False)
    torch.cuda.synchronize()
    refs = [oracle_mod.parflex_full(b.plan(i).cost_matrix().astype(np.float64), STD, WTS, 0.1,
                                    L, fp32=True) for i in range(b.n)]
    _check(b, refs)
    grids = [(-(-(n - 1) // (L - 1)), -(-(m - 1) // (L - 1))) for n, m in shapes]
    b.set_masks(torch.ones(sum(a * c for a, c in grids), dtype=torch.uint8, device="cuda"))
    for use_graph in (False, True):
        b.run(0.1, use_graph=use_graph)
        _check(b, refs)
    dil = []
    for (n, m), r in zip(shapes, refs):
        lab = tiles_on_path(r["wp"], n, m, L).astype(bool)
        p = np.pad(lab, 1)
        d = np.zeros_like(lab)
        for di in range(3):
            for dj in range(3):
                d |= p[di:di + lab.shape[0], dj:dj + lab.shape[1]]
        dil.append(d.reshape(-1))
    masks = torch.from_numpy(np.concatenate(dil).astype(np.uint8)).cuda()
    assert int(masks.sum()) < masks.numel()
    b.set_masks(masks)
    for use_graph in (False, True):
        b.run(0.1, use_graph=use_graph)
        _check(b, refs)
    for i, r in enumerate(refs):
        bc, wp = b.complete(i, 0.1)
        assert bc == r["best_cost"] and same(wp.T, r["wp"])
    b.close()
    from parflexdtw_b200.prune import TileProposer
    pb = pf.PrunedBatch(shapes, L, STD, WTS, 12, proposer=TileProposer(seed=6),
                        threshold=-1e30, precision="fp32")
    pb.load(pairs)
    out, info = pb.run(0.1)
    for (bc, wp), r in zip(out, refs):
        assert bc == r["best_cost"] and same(wp, r["wp"])
    pb.close()


def test_batch_errors():
    with pytest.raises(ValueError):
        Batch([(100, 100)], 100, STD, WTS, 0)  # no features
    with pytest.raises(ValueError):
        Batch([(100, 100)], 100, STD, WTS, 300, precision="fp32")  # beyond the GEMM's K
    with pytest.raises(ValueError):
        Batch([(100, 100)], 100, STD, WTS, 12, warps=5)
    with pytest.raises(ValueError):
        Batch([(100, 100)], 100, [(1, 1), (3, 1)], [1, 1], 12)
    b = Batch([(100, 120)], 50, STD, WTS, 12)
    with pytest.raises(ValueError):
        b.load([(np.zeros((12, 99)), np.zeros((12, 120)))])
    b.close()
    with pytest.raises(ValueError):
        pf.parflex_batch([np.zeros((10, 10))], STD, WTS, 0.1, L=8)
