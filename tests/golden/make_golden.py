"""Generate the golden fixtures in this folder by running the reference itself.

Run in a checkout that has the reference next to it (read-only):

    python tests/golden/make_golden.py --ref <reference checkout>

(or set PARFLEX_REFERENCE to the checkout's path instead of passing --ref).

The reference (``FlexDTW.py``, ``Parflex.py``) is Python + Numba.  It imports
matplotlib and plotly at module top for its plotting helpers; neither is
installed here and neither is on the alignment path, so they are replaced by
empty stub modules before import.  Everything else runs unmodified.

Fixtures written (``np.savez_compressed``):

* ``tile_*.npz``     -- ``FlexDTW.flexdtw`` on one tile: C, D, P, B, best_cost,
  wp (the seeds/shapes of the reference's own tests, ``tests/test_gpu_flexdtw.py``
  lines 20-39, plus other weights and step orders).
* ``tiles_*.npz``    -- ``Parflex.run_flexdtw_on_tiles`` per-tile D, S, B
  (``tests/test_gpu_flexdtw.py`` lines 42-62).
* ``stage2_*.npz``   -- ``Parflex.parflex`` end to end plus every stage-2
  intermediate: edge tensors, valid mask, D_arr/L_arr after propagation and
  after overlap sync, the scan result, and the stitched path.

The reference is never imported at test time; the tests read these files.
"""
from __future__ import annotations

import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))


def _import_reference(ref_dir):
    for name in ("matplotlib", "matplotlib.pyplot", "plotly",
                 "plotly.graph_objects"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.path.insert(0, ref_dir)
    import FlexDTW  # noqa: E402
    import Parflex  # noqa: E402
    return FlexDTW, Parflex


STD_STEPS = [(1, 1), (1, 2), (2, 1)]


def tile_cases(FlexDTW):
    out = {}
    rng = np.random.RandomState(1)
    for H, W in [(5, 6), (17, 19), (48, 50)]:
        C = np.abs(rng.randn(H, W).astype(np.float64)) * 0.1
        out[f"rs1_{H}x{W}"] = (C, STD_STEPS, [2, 3, 3])
    rng = np.random.RandomState(11)
    C = np.abs(rng.randn(37, 29)) * 0.2
    out["rs11_37x29_w125"] = (C, STD_STEPS, [1.25, 3.0, 3.0])
    out["rs11_37x29_w15"] = (C, STD_STEPS, [1.5, 3.0, 3.0])
    out["rs11_37x29_perm"] = (C, [(2, 1), (1, 1), (1, 2)], [3.0, 2.0, 3.0])
    out["rs11_37x29_sub2"] = (C, [(1, 2), (1, 1)], [3.0, 1.5])
    # degenerate shapes: 2 x k and k x 2, and a tile with many exact ties
    rng = np.random.RandomState(12)
    out["rs12_2x9"] = (np.abs(rng.randn(2, 9)), STD_STEPS, [2, 3, 3])
    out["rs12_9x2"] = (np.abs(rng.randn(9, 2)), STD_STEPS, [2, 3, 3])
    out["ties_24x31"] = (np.round(np.abs(rng.randn(24, 31)) * 4) / 4,
                         STD_STEPS, [2, 3, 3])
    res = {}
    for name, (C, steps, weights) in out.items():
        C = np.ascontiguousarray(C, dtype=np.float64)
        bc, wp, D, P, B, _ = FlexDTW.flexdtw(C, steps=np.array(steps),
                                             weights=np.array(weights,
                                                              dtype=np.float64),
                                             buffer=1)
        res[name] = dict(C=C, steps=np.array(steps, dtype=np.int64),
                         weights=np.array(weights, dtype=np.float64),
                         D=D, P=P, B=B, best_cost=np.float64(bc),
                         wp=np.asarray(wp, dtype=np.int64))
    return res


def tiles_case(Parflex):
    rng = np.random.RandomState(2)
    C = np.abs(rng.randn(40, 44).astype(np.float64)) * 0.08
    L = 14
    chunks, Lo, n1, n2 = Parflex.run_flexdtw_on_tiles(
        C, L=L, steps=STD_STEPS, weights=[2, 3, 3], profile_dir=None)
    d = dict(C=C, L=np.int64(L), n1=np.int64(n1), n2=np.int64(n2))
    for (i, j), ch in chunks.items():
        d[f"D_{i}_{j}"] = ch["D"]
        d[f"S_{i}_{j}"] = ch["S"]
        d[f"B_{i}_{j}"] = ch["B"]
        d[f"bounds_{i}_{j}"] = np.array(ch["bounds"], dtype=np.int64)
        d[f"best_{i}_{j}"] = np.float64(ch["best_cost"])
    return d


def stage2_case(Parflex, C, steps, weights, beta, L, feats=None):
    """Everything stage 2 computes, captured with the reference's functions.

    With ``feats=(F1, F2)`` the fixture stores the features instead of C; the
    tests rebuild C bit-exactly with ``workloads.cost_matrix_det``.
    """
    C = np.ascontiguousarray(C, dtype=np.float64)
    L1, L2 = C.shape
    chunks, Lo, n1, n2 = Parflex.run_flexdtw_on_tiles(
        C, L=L, steps=steps, weights=weights, buffer=1, profile_dir=None)
    stage1_params = {"steps": np.array(steps).reshape((-1, 2)),
                     "weights": np.array(weights), "buffer": 1.0}
    tiled = Parflex.build_tiled_metadata(chunks, Lo, n1, n2, C,
                                         stage1_params=stage1_params)
    (edge_Df, esr, esc, eco, elens, crow, ccol, cb, cv) = \
        Parflex._build_edge_data(chunks, n1, n2, Lo)
    vmask = Parflex._build_valid_mask(chunks, n1, n2, Lo)
    D_arr, L_arr, edge_lens = Parflex.propagate_tile_edge_costs(
        chunks, Lo, n1, n2, buffer_param=1, profile_dir=None)
    D_prop, L_prop = D_arr.copy(), L_arr.copy()
    D_arr, L_arr = Parflex.sync_tile_overlap_edges(D_arr, L_arr, edge_lens,
                                                   n1, n2)
    buffer_global = min(L1, L2) * (1 - (1 - beta) * min(L1, L2) / max(L1, L2))
    r = Parflex.stage2_scan_and_stitch(
        tiled, chunks, D_arr.copy(), L_arr.copy(), edge_lens, L1, L2,
        L_block=Lo, buffer_stage2=buffer_global, top_k=1, profile_dir=None,
        backtrace_segments=True)
    best_cost, wp = Parflex.parflex(C, steps, weights, beta, L=L,
                                    profile_dir=None)
    assert np.array_equal(np.asarray(wp).T if np.asarray(wp).size else
                          np.zeros((0, 2), int), r["stitched_wp"]) or \
        np.asarray(wp).size == r["stitched_wp"].size
    seg_keys, seg_paths, seg_norm = [], [], []
    for key, meta in sorted(r["best_per_segment"].items()):
        seg_keys.append([0 if key[0] == "top" else 1, key[1], meta["chunk_i"],
                         meta["chunk_j"], meta["edge"], meta["idx"],
                         meta["global_coord"][0], meta["global_coord"][1]])
        seg_norm.append(meta["norm_cost"])
        p = r["paths_per_segment"][key]["path"]
        seg_paths.append(np.asarray(p, dtype=np.int64).reshape(-1, 2))
    import hashlib
    if feats is not None:
        cdict = dict(F1=feats[0], F2=feats[1],
                     C_sha256=np.frombuffer(hashlib.sha256(C.tobytes())
                                            .digest(), dtype=np.uint8))
    else:
        cdict = dict(C=C)
    d = dict(
        **cdict, steps=np.array(steps, dtype=np.int64),
        weights=np.array(weights, dtype=np.float64), beta=np.float64(beta),
        L=np.int64(L), n1=np.int64(n1), n2=np.int64(n2),
        edge_Df=edge_Df, edge_start_r=esr, edge_start_c=esc,
        edge_Cf_olap=eco, edge_lens=elens, valid_mask=vmask,
        D_prop=D_prop, L_prop=L_prop, D_sync=D_arr, L_sync=L_arr,
        best_cost=np.float64(best_cost),
        best_end=np.array(r["best_end"], dtype=np.int64),
        wp=np.asarray(wp, dtype=np.int64).reshape(2, -1),
        top_D=r["edge_summary"]["top"]["D"], top_L=r["edge_summary"]["top"]["L"],
        right_D=r["edge_summary"]["right"]["D"],
        right_L=r["edge_summary"]["right"]["L"],
        seg_keys=np.array(seg_keys, dtype=np.int64).reshape(-1, 8),
        seg_norm=np.array(seg_norm, dtype=np.float64),
        seg_path_lens=np.array([len(p) for p in seg_paths], dtype=np.int64),
        seg_paths=(np.concatenate(seg_paths) if seg_paths
                   else np.zeros((0, 2), np.int64)),
        tile_S_top=np.stack([chunks[(i, j)]["S"][-1, :].astype(np.int64)
                             .tolist() + [0] * (Lo - chunks[(i, j)]["S"].shape[1])
                             for i in range(n1) for j in range(n2)]),
        tile_S_right=np.stack([chunks[(i, j)]["S"][:, -1].astype(np.int64)
                               .tolist() + [0] * (Lo - chunks[(i, j)]["S"].shape[0])
                               for i in range(n1) for j in range(n2)]),
    )
    return d


def stage2_cases(Parflex):
    from parflexdtw_b200 import workloads as W
    cases = {}
    rng = np.random.RandomState(4)
    cases["rs4_24x28_L11"] = (np.abs(rng.randn(24, 28)) * 0.06, STD_STEPS,
                              [2, 3, 3], 0.1, 11)
    rng = np.random.RandomState(3)
    cases["rs3_16x18_L10"] = (np.abs(rng.randn(16, 18)) * 0.07, STD_STEPS,
                              [2, 3, 3], 0.1, 10)
    rng = np.random.RandomState(2)
    cases["rs2_40x44_L14"] = (np.abs(rng.randn(40, 44)) * 0.08, STD_STEPS,
                              [2, 3, 3], 0.1, 14)
    # chroma-like pairs at small sizes: wide, tall, free start/end, beta sweep
    for seed, (n, m, L, pad, beta, w) in enumerate([
            (150, 190, 40, 0.1, 0.1, (2, 3, 3)),
            (190, 140, 33, 0.1, 0.1, (2, 3, 3)),
            (260, 300, 64, 0.1, 0.5, (1.25, 3, 3)),
            (300, 240, 50, 0.1, 0.9, (1.5, 3, 3)),
            (120, 125, 200, 0.0, 0.1, (2, 3, 3)),   # L larger than both sides
            (97, 131, 32, 0.1, 0.3, (2, 3, 3)),     # ragged last tiles
            (400, 520, 100, 0.1, 0.1, (2, 3, 3)),
    ]):
        r = np.random.default_rng(100 + seed)
        F1, F2 = W.warped_pair(r, n, m, pad_frac=pad)
        cases[f"chroma_s{seed}_{n}x{F2.shape[1]}_L{L}"] = (
            W.cost_matrix_det(F1, F2), STD_STEPS, [float(x) for x in w],
            beta, L, (F1, F2))
    # the 2000 x ~2400, L=500 workload itself
    F1, F2 = W.make_pair(W.CONFIG0)
    cases["config0"] = (W.cost_matrix_det(F1, F2), STD_STEPS,
                        list(W.CONFIG0.weights), W.CONFIG0.beta, W.CONFIG0.L,
                        (F1, F2))
    out = {}
    for name, case in cases.items():
        C, steps, w, beta, L = case[:5]
        feats = case[5] if len(case) > 5 else None
        out[name] = stage2_case(Parflex, C, steps, w, beta, L, feats)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PARFLEX_REFERENCE"),
                    help="path of the reference checkout (default: $PARFLEX_REFERENCE)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("give the reference checkout with --ref or PARFLEX_REFERENCE")
    FlexDTW, Parflex = _import_reference(args.ref)
    for name, d in tile_cases(FlexDTW).items():
        np.savez_compressed(os.path.join(HERE, f"tile_{name}.npz"), **d)
    np.savez_compressed(os.path.join(HERE, "tiles_rs2_40x44_L14.npz"),
                        **tiles_case(Parflex))
    for name, d in stage2_cases(Parflex).items():
        np.savez_compressed(os.path.join(HERE, f"stage2_{name}.npz"), **d)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
