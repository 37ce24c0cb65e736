"""Pin the C oracle to the reference: every golden fixture must be reproduced.

The fixtures hold the reference's own outputs (FlexDTW.flexdtw,
Parflex.run_flexdtw_on_tiles and every stage-2 intermediate of
Parflex.parflex) on seeded inputs; see tests/golden/make_golden.py.
"""
import numpy as np
import pytest

from golden_util import load, names


@pytest.mark.parametrize("name", names("tile"))
def test_tile_dp_matches_reference(oracle_mod, name):
    g = load("tile", name)
    best, wp, D, P, B = oracle_mod.flexdtw(g["C"], g["steps"], g["weights"], 1)
    assert np.array_equal(D, g["D"])          # bit-exact FP64
    assert np.array_equal(P, g["P"])
    assert np.array_equal(B, g["B"])
    assert best == g["best_cost"]
    assert np.array_equal(wp, g["wp"])


def test_tiles_match_reference(oracle_mod):
    g = load("tiles", "rs2_40x44_L14")
    C, L = g["C"], int(g["L"])
    hop = L - 1
    for i in range(int(g["n1"])):
        for j in range(int(g["n2"])):
            s1, e1, s2, e2 = g[f"bounds_{i}_{j}"]
            assert (s1, s2) == (i * hop, j * hop)
            best, wp, D, P, B = oracle_mod.flexdtw(C[s1:e1, s2:e2],
                                                   [(1, 1), (1, 2), (2, 1)],
                                                   [2, 3, 3])
            assert np.array_equal(D, g[f"D_{i}_{j}"])
            assert np.array_equal(P, g[f"S_{i}_{j}"])
            assert np.array_equal(B, g[f"B_{i}_{j}"])
            assert best == g[f"best_{i}_{j}"]


def _inf_equal(a, b):
    return np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("name", names("stage2"))
def test_stage2_matches_reference(oracle_mod, name):
    g = load("stage2", name)
    r = oracle_mod.parflex_full(g["C"], g["steps"], g["weights"],
                                float(g["beta"]), int(g["L"]), threads=2)
    assert (r["n1"], r["n2"]) == (int(g["n1"]), int(g["n2"]))
    assert _inf_equal(r["edge_Df"], g["edge_Df"])
    assert np.array_equal(r["edge_start_r"], g["edge_start_r"])
    assert np.array_equal(r["edge_start_c"], g["edge_start_c"])
    assert np.array_equal(r["edge_Cf_olap"], g["edge_Cf_olap"])
    assert np.array_equal(r["edge_lens"], g["edge_lens"])
    assert np.array_equal(r["valid_mask"], g["valid_mask"])
    assert _inf_equal(r["D_prop"], g["D_prop"])
    assert _inf_equal(r["L_prop"], g["L_prop"])
    assert _inf_equal(r["D_arr"], g["D_sync"])
    assert _inf_equal(r["L_arr"], g["L_sync"])
    assert _inf_equal(r["top_D"], g["top_D"])
    assert _inf_equal(r["top_L"], g["top_L"])
    assert _inf_equal(r["right_D"], g["right_D"])
    assert _inf_equal(r["right_L"], g["right_L"])
    assert r["best_cost"] == float(g["best_cost"])
    assert r["best_end"] == tuple(int(x) for x in g["best_end"])
    assert np.array_equal(r["wp"], g["wp"])
    # per-segment winners of the edge scan
    for row, norm in zip(g["seg_keys"], g["seg_norm"]):
        et, si, ci, cj, e, ix, gr, gc = (int(x) for x in row)
        assert r["seg_best_norm"][et, si] == norm
        assert tuple(r["seg_best_meta"][et, si]) == (ci, cj, e, ix, gr, gc)


def test_oracle_cost_fma_is_the_fma_chain():
    """oracle_cost_fma: C = 1 - (fma chain over the features in order); it
    differs from the separately rounded cost by a few ulps at most, and
    equals an independent evaluation of the chain (math.fma where Python has
    it, else the exact rational product-sum rounded once per step)."""
    import math
    from fractions import Fraction
    from parflexdtw_b200 import workloads as W
    from oracle import oracle as O
    rng = np.random.default_rng(8)
    F1, F2 = W.warped_pair(rng, 40, 35, d=7, noise=0.1, latent="gaussian")
    C = O.cost_matrix_fma(F1, F2)
    C0 = W.cost_matrix_det(F1, F2)
    assert np.abs(C - C0).max() < 1e-14
    A, B = W.l2norm(F1), W.l2norm(F2)

    def fma(a, b, c):
        if hasattr(math, "fma"):
            return math.fma(a, b, c)
        return float(Fraction(a) * Fraction(b) + Fraction(c))  # one rounding

    for i, j in [(0, 0), (3, 17), (39, 34), (20, 5)]:
        acc = A[0, i] * B[0, j]
        for f in range(1, A.shape[0]):
            acc = fma(A[f, i], B[f, j], acc)
        assert C[i, j] == 1.0 - acc
