"""Device path vs the reference (golden fixtures) and vs the C oracle.

Parity bar (plain FP64 form): every integer output (paths, start encodings,
backpointers, valid masks, indices) bit-exact, and every FP64 output
(D, accumulated costs, lengths, best cost) bit-exact as well -- the device
evaluates the same IEEE operations in the same order as the reference, so the
tolerance written here is zero.
"""
import numpy as np
import pytest

from golden_util import load, names

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover - CPU container
    pytest.skip("needs a CUDA device", allow_module_level=True)

import parflexdtw_b200 as pf  # noqa: E402
from parflexdtw_b200 import workloads as W  # noqa: E402

STD = [(1, 1), (1, 2), (2, 1)]


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


# ---------------------------------------------------------------------------
# single tile: FlexDTW.flexdtw golden vectors
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", names("tile"))
def test_tile_dp_golden(name):
    g = load("tile", name)
    C = g["C"]
    Cd = torch.from_numpy(C).cuda()
    best, wp, D, P, B, debug = pf.flexdtw_chunk_from_global_C(
        Cd, C.shape[1], 0, C.shape[0], 0, C.shape[1], g["steps"], g["weights"], 1)
    assert same(D, g["D"])
    assert same(P, g["P"])
    assert same(B, g["B"])
    assert best == g["best_cost"]
    assert same(wp, g["wp"])


def test_tile_offsets_in_global_C(oracle_mod):
    """A tile cut out of a larger C (64-bit offsets, ldc != W)."""
    rng = np.random.RandomState(7)
    C = np.abs(rng.randn(300, 410)) * 0.3
    Cd = torch.from_numpy(C).cuda()
    for (r0, r1, c0, c1) in [(0, 300, 0, 410), (37, 211, 101, 409), (299 - 64, 299, 5, 70)]:
        _, _, D, P, B, _ = pf.flexdtw_chunk_from_global_C(Cd, 410, r0, r1, c0, c1, STD,
                                                         [2, 3, 3])
        _, _, Do, Po, Bo = oracle_mod.flexdtw(C[r0:r1, c0:c1], STD, [2, 3, 3])
        assert same(D, Do) and same(P, Po) and same(B, Bo)


def test_tile_shapes_sweep(oracle_mod):
    """Every strip / lag / ragged-edge regime of the wavefront schedule."""
    rng = np.random.RandomState(8)
    for R, Wd in [(2, 2), (2, 40), (40, 2), (31, 33), (32, 32), (33, 31), (64, 65),
                  (65, 64), (97, 300), (300, 97), (257, 255), (511, 513)]:
        C = np.abs(rng.randn(R, Wd)) * 0.25
        Cd = torch.from_numpy(C).cuda()
        _, wp, D, P, B, _ = pf.flexdtw_chunk_from_global_C(Cd, Wd, 0, R, 0, Wd, STD,
                                                          [2, 3, 3])
        bo, wpo, Do, Po, Bo = oracle_mod.flexdtw(C, STD, [2, 3, 3])
        assert same(D, Do), (R, Wd)
        assert same(P, Po), (R, Wd)
        assert same(B, Bo), (R, Wd)
        assert same(wp, wpo), (R, Wd)


def test_tiles_golden():
    g = load("tiles", "rs2_40x44_L14")
    chunks, Lo, n1, n2 = pf.run_flexdtw_on_tiles(g["C"], L=int(g["L"]), steps=STD,
                                                 weights=[2, 3, 3], profile_dir=None)
    assert (Lo, n1, n2) == (int(g["L"]), int(g["n1"]), int(g["n2"]))
    for (i, j), ch in chunks.items():
        assert tuple(ch["bounds"]) == tuple(g[f"bounds_{i}_{j}"])
        assert same(ch["D"], g[f"D_{i}_{j}"])
        assert same(ch["S"], g[f"S_{i}_{j}"])
        assert same(ch["B"], g[f"B_{i}_{j}"])
        assert ch["best_cost"] == g[f"best_{i}_{j}"]


# ---------------------------------------------------------------------------
# stage 2: every intermediate against the reference's own values
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", names("stage2"))
def test_stage2_golden(name):
    g = load("stage2", name)
    C = g["C"]
    N, M = C.shape
    Lb = int(g["L"])
    plan = pf.Plan(N, M, Lb, g["steps"], g["weights"])
    Cd = torch.from_numpy(C).cuda()
    plan.stage1(Cd)
    plan.propagate(Cd, snapshot=True)
    plan.scan(float(g["beta"]))
    plan.stitch()
    best, end, found, n = plan.result()
    el = g["edge_lens"]
    eD = plan.host("EDGE_D")
    assert same(eD, g["edge_Df"])
    P = plan.host("EDGE_P").astype(np.int64)
    sr = np.where(P < 0, -P, 0)
    sc = np.where(P > 0, P, 0)
    mask = np.zeros_like(P, dtype=bool)
    for i in range(el.shape[0]):
        for j in range(el.shape[1]):
            mask[i, j, 0, :el[i, j, 0]] = True
            mask[i, j, 1, :el[i, j, 1]] = True
    assert same(np.where(mask, sr, 0), g["edge_start_r"])
    assert same(np.where(mask, sc, 0), g["edge_start_c"])
    assert same(plan.host("EDGE_CF"), g["edge_Cf_olap"])
    assert same(plan.host("VALID").astype(bool), g["valid_mask"])
    assert same(plan.host("D_PROP"), g["D_prop"])
    assert same(plan.host("L_PROP"), g["L_prop"])
    assert same(plan.host("D_ARR"), g["D_sync"])
    assert same(plan.host("L_ARR"), g["L_sync"])
    assert same(plan.host("TOP_D"), g["top_D"])
    assert same(plan.host("TOP_L"), g["top_L"])
    assert same(plan.host("RIGHT_D"), g["right_D"])
    assert same(plan.host("RIGHT_L"), g["right_L"])
    assert best == float(g["best_cost"])
    assert end == tuple(int(x) for x in g["best_end"])
    assert same(plan.path(n).T, g["wp"])


@pytest.mark.parametrize("name", names("stage2"))
def test_parflex_api_golden(name):
    g = load("stage2", name)
    best, wp = pf.parflex(g["C"], g["steps"], g["weights"], float(g["beta"]),
                          L=int(g["L"]), profile_dir=None)
    assert best == float(g["best_cost"])
    assert wp.dtype == np.int64 and wp.shape[0] == 2
    assert same(wp, g["wp"])


@pytest.mark.parametrize("name", ["rs4_24x28_L11", "chroma_s2_260x323_L64", "config0"])
def test_backtrace_segments_golden(name):
    g = load("stage2", name)
    C = g["C"]
    Cd = torch.from_numpy(C).cuda()
    tr = {"C_shape": C.shape, "L_block": int(g["L"]), "n_row": int(g["n1"]),
          "n_col": int(g["n2"])}
    chunks, Lo, n1, n2 = pf.run_flexdtw_on_tiles(None, int(g["L"]), g["steps"],
                                                 g["weights"], profile_dir=None, C_dev=Cd)
    tr["chunks_dict"] = chunks
    tr["C_dev"] = Cd
    r = pf.run_stage2_from_tiled(tr, beta=float(g["beta"]), backtrace_segments=True)
    bps = r["best_per_segment"]
    paths = r["paths_per_segment"]
    off = 0
    names_ = ["top", "right"]
    assert len(bps) == g["seg_keys"].shape[0]
    for row, norm, ln in zip(g["seg_keys"], g["seg_norm"], g["seg_path_lens"]):
        et, si, ci, cj, e, ix, gr, gc = (int(x) for x in row)
        meta = bps[(names_[et], si)]
        assert (meta["chunk_i"], meta["chunk_j"], meta["edge"], meta["idx"]) == (ci, cj, e, ix)
        assert meta["global_coord"] == (gr, gc)
        assert meta["norm_cost"] == norm
        ref = g["seg_paths"][off:off + ln]
        off += ln
        assert same(np.array(paths[(names_[et], si)]["path"]).reshape(-1, 2), ref)
    # the best path is still the result after the per-segment walks
    assert same(r["stitched_wp"].T, g["wp"])
    assert r["best_cost"] == float(g["best_cost"])


# ---------------------------------------------------------------------------
# random sweeps against the oracle
# ---------------------------------------------------------------------------
CASES = [
    # (n, m_core, L, pad, beta, weights)
    (700, 800, 128, 0.1, 0.1, (2, 3, 3)),
    (800, 650, 100, 0.1, 0.1, (2, 3, 3)),
    (1500, 1800, 300, 0.1, 0.3, (1.25, 3, 3)),
    (1000, 1000, 2000, 0.0, 0.1, (1.5, 3, 3)),   # one tile, L > N, M
    (333, 1200, 90, 0.1, 0.1, (2, 3, 3)),        # very wide
    (1200, 333, 90, 0.1, 0.1, (2, 3, 3)),        # very tall
    (3000, 3600, 500, 0.1, 0.1, (2, 3, 3)),      # config-0 geometry, other seed
    (2049, 2050, 1025, 0.1, 0.1, (2, 3, 3)),     # L with 16-warp CTAs
]


@pytest.mark.parametrize("case", CASES)
def test_random_pairs_vs_oracle(case, oracle_mod):
    n, m, Lb, pad, beta, w = case
    rng = np.random.default_rng(hash(case) % (2 ** 32))
    F1, F2 = W.warped_pair(rng, n, m, pad_frac=pad)
    C = W.cost_matrix_det(F1, F2)
    ref = oracle_mod.parflex_full(C, STD, w, beta, Lb)
    best, wp = pf.parflex(C, STD, w, beta, L=Lb, profile_dir=None)
    assert best == ref["best_cost"]
    assert same(wp, ref["wp"])


def test_permuted_and_partial_steps_vs_oracle(oracle_mod):
    rng = np.random.default_rng(5)
    F1, F2 = W.warped_pair(rng, 600, 700, pad_frac=0.1)
    C = W.cost_matrix_det(F1, F2)
    for steps, w in [([(2, 1), (1, 1), (1, 2)], [3, 2, 3]),
                     ([(1, 2), (1, 1)], [3.0, 1.5]),
                     ([(1, 1)], [1.0])]:
        ref = oracle_mod.parflex_full(C, steps, w, 0.1, 150)
        best, wp = pf.parflex(C, steps, w, 0.1, L=150, profile_dir=None)
        assert best == ref["best_cost"], steps
        assert same(wp, ref["wp"]), steps


def test_features_pipeline_vs_oracle(oracle_mod):
    """tiled_stage1_from_features -> run_stage2_from_tiled; the device cost
    matrix equals the fixed-order host restatement bit for bit."""
    rng = np.random.default_rng(11)
    F1, F2 = W.warped_pair(rng, 2500, 3000, pad_frac=0.1)
    C_host = W.cost_matrix_det(F1, F2)
    C_none, tr = pf.tiled_stage1_from_features(F1, F2, steps=STD, weights=[2, 3, 3],
                                               beta=0.1, L=400)
    assert C_none is None
    assert same(tr["C_dev"].cpu().numpy(), C_host)
    r = pf.run_stage2_from_tiled(tr, beta=0.1)
    ref = oracle_mod.parflex_full(C_host, STD, [2, 3, 3], 0.1, 400)
    assert r["best_cost"] == ref["best_cost"]
    assert r["best_end"] == ref["best_end"]
    assert same(r["stitched_wp"].T, ref["wp"])
    assert same(r["D_arr"], ref["D_arr"])
    assert same(r["L_arr"], ref["L_arr"])
    assert same(r["edge_summary"]["top"]["D"], ref["top_D"])
    assert same(r["edge_summary"]["right"]["L"], ref["right_L"])
    # lazily materialised per-tile records
    ch = tr["chunks_dict"][(1, 2)]
    s1, e1, s2, e2 = ch["bounds"]
    _, _, Do, Po, Bo = oracle_mod.flexdtw(C_host[s1:e1, s2:e2], STD, [2, 3, 3])
    assert same(ch["D"], Do) and same(ch["S"], Po) and same(ch["B"], Bo)
    assert same(ch["C"], C_host[s1:e1, s2:e2])
    blk = tr["blocks"][0]
    assert blk["bi"] == 0 and blk["bj"] == 0


def test_no_endpoint_raises():
    rng = np.random.default_rng(3)
    F1, F2 = W.warped_pair(rng, 200, 200)
    C = W.cost_matrix_det(F1, F2)
    with pytest.raises(ValueError, match="No valid endpoint"):
        pf.parflex(C, STD, [2, 3, 3], 1.0, L=50, profile_dir=None)


def test_bad_arguments_raise():
    C = np.abs(np.random.RandomState(0).randn(50, 60))
    with pytest.raises(ValueError):
        pf.parflex(C, [(1, 0), (0, 1)], [1, 1], 0.1, L=20, profile_dir=None)
    with pytest.raises(ValueError):
        pf.parflex(C, STD, [2, 3, 3], 0.1, L=20, profile_dir=None, use_gpu=False)
    with pytest.raises(ValueError):
        pf.parflex(C, STD, [2, 3], 0.1, L=20, profile_dir=None)


def test_profile_csv(tmp_path):
    rng = np.random.default_rng(4)
    F1, F2 = W.warped_pair(rng, 300, 320)
    C = W.cost_matrix_det(F1, F2)
    pf.parflex(C, STD, [2, 3, 3], 0.1, L=100, profile_dir=str(tmp_path))
    text = (tmp_path / "parflex_end_to_end_phases.csv").read_text()
    assert "stage1_chunk_flexdtw_all_tiles" in text


@pytest.mark.slow
def test_config1_full_size_vs_oracle(oracle_mod):
    """The 30000 x ~37000, L=4000 workload end to end, bit-exact."""
    spec = W.CONFIG1
    F1, F2 = W.make_pair(spec)
    C_dev = pf.cost_matrix_from_features_gpu(F1, F2)
    best, wp = pf.parflex(C_dev, spec.steps, spec.weights, spec.beta, L=spec.L,
                          profile_dir=None)
    C = C_dev.cpu().numpy()
    del C_dev
    ref = oracle_mod.parflex_full(C, spec.steps, spec.weights, spec.beta, spec.L)
    assert best == ref["best_cost"]
    assert same(wp, ref["wp"])


# ---------------------------------------------------------------------------
# tile-skewed cost layout: relayout of a row-major C and the fused features
# path give the same stage-1 products, for every strip / block regime
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("Lb", [2, 3, 5, 17, 63, 64, 65, 127, 129, 300])
def test_small_tile_lengths_vs_oracle(Lb, oracle_mod):
    rng = np.random.default_rng(1000 + Lb)
    F1, F2 = W.warped_pair(rng, 260, 310, pad_frac=0.1)
    C = W.cost_matrix_det(F1, F2)
    ref = oracle_mod.parflex_full(C, STD, [2, 3, 3], 0.1, Lb)
    plan = pf.Plan(C.shape[0], C.shape[1], Lb, STD, [2, 3, 3])
    Cd = torch.from_numpy(C).cuda()
    plan.run(Cd, 0.1)
    best, end, found, n = plan.result()
    assert same(plan.host("EDGE_D"), ref["edge_Df"])
    assert same(plan.host("EDGE_P"), ref["edge_S"])
    assert same(plan.host("D_ARR"), ref["D_arr"])
    assert best == ref["best_cost"] and end == ref["best_end"]
    assert same(plan.path(n).T, ref["wp"])


@pytest.mark.parametrize("Lb", [64, 1000, 2500])
def test_fused_and_relayout_cost_agree(Lb, oracle_mod):
    rng = np.random.default_rng(77 + Lb)
    F1, F2 = W.warped_pair(rng, 2600, 2900, pad_frac=0.1)
    C = W.cost_matrix_det(F1, F2)
    N, M = C.shape
    pa = pf.Plan(N, M, Lb, STD, [2, 3, 3])
    pb = pf.Plan(N, M, Lb, STD, [2, 3, 3])
    pa.load_features(torch.from_numpy(F1).cuda(), torch.from_numpy(F2).cuda())
    pb.load_cost(torch.from_numpy(C).cuda())
    for p in (pa, pb):
        p.run(None, 0.1)
    for name in ("EDGE_D", "EDGE_P", "BACKPTR", "EDGE_CF", "D_ARR", "L_ARR"):
        assert same(pa.host(name), pb.host(name)), name
    ra, rb = pa.result(), pb.result()
    assert ra == rb
    ref = oracle_mod.parflex_full(C, STD, [2, 3, 3], 0.1, Lb)
    assert ra[0] == ref["best_cost"]
    assert same(pa.path(ra[3]).T, ref["wp"])


def test_plan_reuse_across_pairs(oracle_mod):
    """One plan, two different cost matrices in a row (no stale state)."""
    rng = np.random.default_rng(9)
    pairs = [W.warped_pair(rng, 700, 760, pad_frac=0.1) for _ in range(2)]
    plan = pf.Plan(700, pairs[0][1].shape[1], 200, STD, [2, 3, 3])
    for F1, F2 in pairs:
        if F2.shape[1] != plan.M:
            F2 = F2[:, :plan.M] if F2.shape[1] > plan.M else np.pad(
                F2, ((0, 0), (0, plan.M - F2.shape[1])), constant_values=0.1)
        C = W.cost_matrix_det(F1, F2)
        plan.load_features(torch.from_numpy(F1).cuda(), torch.from_numpy(F2).cuda())
        plan.run(None, 0.1)
        best, end, found, n = plan.result()
        ref = oracle_mod.parflex_full(C, STD, [2, 3, 3], 0.1, 200)
        assert best == ref["best_cost"]
        assert same(plan.path(n).T, ref["wp"])


# fewer tiles than SMs, more than half: the largest tiles run on 2-CTA
# clusters and the rest on single CTAs in a second stream, at the same time
@pytest.mark.parametrize("shape,Lb,fp32", [((600, 700), 64, False), ((900, 1000), 100, False),
                                          ((600, 700), 64, True), ((300, 320), 300, False)])
def test_cluster_and_single_tiles_vs_oracle(shape, Lb, fp32, oracle_mod):
    rng = np.random.default_rng(shape[0] + Lb)
    F1, F2 = W.warped_pair(rng, shape[0], shape[1], pad_frac=0.1)
    C = W.cost_matrix_det(F1, F2)
    if fp32:
        C = C.astype(np.float32).astype(np.float64)
    ref = oracle_mod.parflex_full(C, STD, [2, 3, 3], 0.1, Lb, fp32=fp32)
    plan = pf.Plan(C.shape[0], C.shape[1], Lb, STD, [2, 3, 3],
                   precision="fp32" if fp32 else "fp64")
    Cd = torch.from_numpy(C).cuda()
    for _ in range(2):  # the second run reuses the plan's streams and queues
        plan.run(Cd, 0.1)
        best, end, found, n = plan.result()
        assert same(plan.host("EDGE_D"), ref["edge_Df"])
        assert same(plan.host("EDGE_P"), ref["edge_S"])
        assert best == ref["best_cost"] and end == ref["best_end"]
        assert same(plan.path(n).T, ref["wp"])
    plan.close()


# the untiled FlexDTW (one device tile over the whole matrix), with the
# global buffer ParFlex's stage 2 uses
@pytest.mark.parametrize("n,m,beta", [(300, 360, 0.1), (900, 700, 0.3), (64, 2000, 0.1)])
def test_global_flexdtw_vs_oracle(n, m, beta, oracle_mod):
    rng = np.random.default_rng(n + m)
    F1, F2 = W.warped_pair(rng, n, m, pad_frac=0.1)
    C = W.cost_matrix_det(F1, F2)
    buf = pf.buffer_global(C.shape[0], C.shape[1], beta)
    best, wp, D, P, B, debug = pf.flexdtw(C, STD, [2, 3, 3], buf)
    rbest, rwp, rD, rP, rB = oracle_mod.flexdtw(C, STD, [2, 3, 3], buf)
    assert best == rbest
    assert same(wp, rwp)
    assert same(D, rD) and same(P, rP) and same(B, rB)


def test_host_cost_matrix_staged_upload():
    """A host cost matrix above one staging chunk goes to the device through
    the double-buffered staged upload: bit for bit the matrix, on consecutive
    calls (the chunks are reused once their transfers are done), and the
    drop-in call on it returns the plan path's result."""
    from parflexdtw_b200.parflex import _STAGE_ELEMS, cost_matrix_to_gpu
    rng = np.random.default_rng(11)
    N, M = 6100, 5600  # 34.2 M elements: one full chunk and a partial one
    assert _STAGE_ELEMS < N * M < 2 * _STAGE_ELEMS
    for _ in range(2):
        C = rng.random((N, M))
        got = cost_matrix_to_gpu(C)
        assert got.dtype == torch.float64 and tuple(got.shape) == (N, M)
        assert torch.equal(got.cpu(), torch.from_numpy(C))
    F1, F2 = W.warped_pair(np.random.default_rng(3), 6000, 5900)
    C = pf.cost_matrix_from_features_gpu(F1, F2).cpu().numpy()
    assert C.size > _STAGE_ELEMS
    b_host, wp_host = pf.parflex(C, STD, [2.0, 3.0, 3.0], 0.1, L=2000, profile_dir=None)
    b_dev, wp_dev = pf.parflex(torch.from_numpy(C).cuda(), STD, [2.0, 3.0, 3.0], 0.1,
                               L=2000, profile_dir=None)
    assert b_host == b_dev and np.array_equal(wp_host, wp_dev)
