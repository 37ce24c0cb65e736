"""FP32 form (PFX_FP32 plans): FP32 stage-1 DP and the BF16 tensor-core cost.

Parity bar:
  * DP: bit-exact against the oracle's FP32 form (oracle_tile_dp_f32 +
    FP64 stage 2 on widened values) fed the same FP32 cost -- paths, best
    cost, propagated arrays: tolerance zero.
  * Tensor-core cost: against a plain PyTorch reference of the same op on
    the kernel's own bf16 operands (exact products summed in FP64):
    |dC| <= 1e-6, the FP32 accumulation error of <= 256 products of
    magnitude <= 1; the operands themselves are checked against an
    independent round-to-nearest of the FP64-normalised features.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

from parflexdtw_b200 import workloads as W  # noqa: E402
from parflexdtw_b200.plan import Plan  # noqa: E402

STD = [(1, 1), (1, 2), (2, 1)]
WTS = [2.0, 3.0, 3.0]
GEMM_TOL = 1e-6  # measured 2.0e-7 on B200; torch's own FP32 GEMM: 2.3e-7


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


def _run(plan, beta):
    plan.stage1()
    plan.propagate()
    plan.scan(beta)
    plan.stitch()
    best, end, found, n = plan.result()
    return best, end, plan.path(n)


@pytest.mark.parametrize("shape,Lb", [((900, 1000), 300), ((1500, 1200), 500),
                                       ((333, 410), 64), ((2100, 2600), 1000)])
def test_fp32_dp_vs_oracle(shape, Lb, oracle_mod):
    rng = np.random.default_rng(shape[0] + Lb)
    F1, F2 = W.warped_pair(rng, shape[0], shape[1], pad_frac=0.1)
    C = W.cost_matrix_det(F1, F2)
    p = Plan(C.shape[0], C.shape[1], Lb, STD, WTS, precision="fp32")
    p.load_cost(torch.from_numpy(C).cuda())  # rounded to FP32 on the device
    best, end, wp = _run(p, 0.1)
    ref = oracle_mod.parflex_full(C, STD, WTS, 0.1, Lb, fp32=True)
    assert same(p.cost_matrix(), C.astype(np.float32))
    assert best == ref["best_cost"]
    assert end == ref["best_end"]
    assert same(wp.T, ref["wp"])
    assert same(p.host("D_ARR"), ref["D_arr"])
    assert same(p.host("EDGE_D"), ref["edge_Df"])


def test_fp32_cost_from_float_matrix(oracle_mod):
    rng = np.random.default_rng(4)
    C = (np.abs(rng.standard_normal((700, 820))) * 0.4).astype(np.float32)
    p = Plan(700, 820, 200, STD, WTS, precision="fp32")
    p.load_cost(torch.from_numpy(C).cuda())
    best, end, wp = _run(p, 0.1)
    ref = oracle_mod.parflex_full(C.astype(np.float64), STD, WTS, 0.1, 200, fp32=True)
    assert best == ref["best_cost"] and same(wp.T, ref["wp"])


def test_fp32_tile_dp_vs_oracle_steps(oracle_mod):
    """Generic (non-standard order / subset) steps in the FP32 DP."""
    rng = np.random.default_rng(6)
    F1, F2 = W.warped_pair(rng, 600, 700, pad_frac=0.1)
    C = W.cost_matrix_det(F1, F2)
    for steps, w in [([(2, 1), (1, 1), (1, 2)], [3, 2, 3]), ([(1, 2), (1, 1)], [3.0, 1.5])]:
        p = Plan(C.shape[0], C.shape[1], 150, steps, w, precision="fp32")
        p.load_cost(torch.from_numpy(C).cuda())
        best, end, wp = _run(p, 0.1)
        ref = oracle_mod.parflex_full(C, steps, w, 0.1, 150, fp32=True)
        assert best == ref["best_cost"], steps
        assert same(wp.T, ref["wp"]), steps


def _bf16_rn(x):
    """FP64 -> nearest bf16 (ties to even), returned as FP64 (normal range)."""
    b = np.ascontiguousarray(x, dtype=np.float64).view(np.uint64)
    drop = np.uint64(45)
    mask = (np.uint64(1) << drop) - np.uint64(1)
    half = np.uint64(1) << np.uint64(44)
    low = b & mask
    lsb = (b >> drop) & np.uint64(1)
    up = (low > half) | ((low == half) & (lsb == np.uint64(1)))
    return ((b & ~mask) + (up.astype(np.uint64) << drop)).view(np.float64)


def _normalised(F):
    n = np.sqrt(np.sum(F * F, axis=0, keepdims=True))
    return F / n


@pytest.mark.parametrize("d,shape,Lb", [(128, (1000, 1300), 1000), (128, (2500, 1900), 1000),
                                         (64, (700, 500), 300), (200, (600, 900), 256),
                                         (150, (500, 700), 256),
                                         (12, (400, 450), 128)])
def test_tensor_core_cost_vs_torch(d, shape, Lb):
    rng = np.random.default_rng(d + shape[0])
    F1, F2 = W.warped_pair(rng, shape[0], shape[1], d=d, noise=0.1, latent="gaussian")
    N, M = F1.shape[1], F2.shape[1]
    p = Plan(N, M, Lb, STD, WTS, precision="fp32")
    p.load_features(torch.from_numpy(F1).cuda(), torch.from_numpy(F2).cuda())
    torch.cuda.synchronize()
    got = p.cost_matrix()
    # the operands: L2-normalised in FP64, rounded to nearest bf16
    feats = p.view("FEAT_BF16").float().double()
    A, B = feats[:N, :d], feats[N:, :d]
    assert torch.all(feats[:, d:] == 0)
    exp_a = _bf16_rn(_normalised(F1)).T
    nrm_diff = np.abs(A.cpu().numpy() - exp_a)
    # FP64 norms may differ from numpy's in the last bit: allow one bf16 ulp
    assert nrm_diff.max() <= 2.0 ** -8 * np.abs(exp_a).max()
    assert (nrm_diff > 0).mean() < 1e-3
    # plain PyTorch reference of the same op: exact products, FP64 sum
    ref = (1.0 - A @ B.T).cpu().numpy()
    err = np.abs(got.astype(np.float64) - ref)
    assert err.max() <= GEMM_TOL, err.max()


def test_fp32_form_from_features_vs_oracle(oracle_mod):
    """Features -> tensor-core cost -> FP32 DP -> stage 2, against the
    oracle's FP32 form fed the device's own FP32 cost."""
    rng = np.random.default_rng(21)
    F1, F2 = W.warped_pair(rng, 3000, 3500, d=128, noise=0.1, latent="gaussian")
    p = Plan(F1.shape[1], F2.shape[1], 1000, STD, WTS, precision="fp32")
    p.load_features(torch.from_numpy(F1).cuda(), torch.from_numpy(F2).cuda())
    best, end, wp = _run(p, 0.1)
    C32 = p.cost_matrix()
    ref = oracle_mod.parflex_full(C32.astype(np.float64), STD, WTS, 0.1, 1000, fp32=True)
    assert best == ref["best_cost"]
    assert same(wp.T, ref["wp"])
    # and the FP64 form on the FP64 cost takes (here) the same path
    C64 = W.cost_matrix_det(F1, F2)
    ref64 = oracle_mod.parflex_full(C64, STD, WTS, 0.1, 1000)
    assert abs(best - ref64["best_cost"]) <= 1e-2 * abs(ref64["best_cost"])


def test_fp32_plan_errors():
    p = Plan(300, 300, 100, STD, WTS, precision="fp32")
    with pytest.raises(ValueError):
        p.stage1()  # no cost loaded
    f = torch.zeros((300, 12), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        p.load_features(torch.zeros((300, 300), dtype=torch.float64, device="cuda"), f)
    with pytest.raises(ValueError):
        Plan(300, 300, 100, STD, WTS, precision="fp16")


NEAR_TIE_TOL = 5e-3  # relative; the largest gap measured over all 2048 pairs was 2.7e-3


def test_fp32_form_divergent_paths_are_near_ties():
    """The FP32 form (BF16 tensor-core cost, FP32 DP) does not reproduce the
    FP64 path on every pair.  Its rule: a path that differs must be a near
    tie -- re-scored under the FP64 cost (the reference's normalised path
    cost, FlexDTW.py:326-370), it lies within NEAR_TIE_TOL (relative) of the
    FP64 form's best cost.  Sample: the first 32 pairs of the precision
    workload (N, M ~ U(1000, 8000), 128-d Gaussian latents, L = 1000)."""
    from parflexdtw_b200 import precision as PR
    from parflexdtw_b200.batch import Batch
    pairs = W.make_precision_batch(W.PRECISION2048, n_pairs=32)
    shapes = [(F1.shape[1], F2.shape[1]) for F1, F2 in pairs]
    res = {}
    for prec in ("fp32", "fp64"):
        b = Batch(shapes, 1000, STD, WTS, 128, precision=prec)
        b.load(pairs)
        b.run(0.1, use_graph=False)
        best, end, lens = b.results()
        res[prec] = (best, end, b.paths(lens))
        b.close()
    (b32, e32, p32), (b64, e64, p64) = res["fp32"], res["fp64"]
    rep = PR.compare_results(pairs, b32, p32, b64, p64, STD, WTS, e32[:, 6], e64[:, 6])
    print(rep)
    assert rep["pairs"] == 32
    assert rep["best_cost_rel_err_max"] < 0.2
    if rep["divergent_pairs"]:
        assert rep["divergent_fp32_path_fp64_score_rel_gap_max"] <= NEAR_TIE_TOL, rep
        # the FP64 path re-scored the same way reproduces the FP64 best cost
        assert rep["divergent_fp64_path_rescore_rel_dev_max"] < 1e-9, rep
    for i in range(32):
        s32 = PR.path_score(*pairs[i], p32[i], STD, WTS)
        assert abs(s32 - b64[i]) / b64[i] <= NEAR_TIE_TOL, (i, s32, b64[i])
