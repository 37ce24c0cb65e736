"""Precision report of the FP32 form against the FP64 plain form.

For a batch aligned in both forms (same pairs, same tile length):

* cost-matrix error: max / mean |C_fp32 - C_fp64| over the cells of sample
  pairs, read back from both forms' device cost slabs;
* accumulated-cost error: |best_fp32 - best_fp64| / |best_fp64| per pair;
* path agreement: the fraction of pairs whose stitched paths are identical;
* near-tie evidence for every divergent pair: the FP32 form's path re-scored
  under the FP64 cost (FlexDTW path cost: the start cell's cost plus each
  later cell's cost times its step weight, over the path length
  (r_end + c_end) - (r_start + c_start), FlexDTW.py:326-370) against the
  FP64 optimum, as a relative gap; and the same re-scoring of the FP64 path,
  which reproduces the FP64 optimum up to summation order.
"""
from __future__ import annotations

import numpy as np

from .workloads import l2norm


def _cost_along(F1, F2, wp):
    """FP64 cost (fixed order f = 0..d-1, as the plain form) at path points."""
    A = l2norm(np.asarray(F1, dtype=np.float64))[:, wp[:, 0]]
    B = l2norm(np.asarray(F2, dtype=np.float64))[:, wp[:, 1]]
    acc = A[0] * B[0]
    for k in range(1, A.shape[0]):
        acc = acc + A[k] * B[k]
    return 1.0 - acc


def path_score(F1, F2, wp, steps, weights):
    """Normalised FP64 cost of a (K, 2) path (start first)."""
    wp = np.asarray(wp, dtype=np.int64)
    if wp.shape[0] < 2:
        return float("nan")
    c = _cost_along(F1, F2, wp)
    d = np.diff(wp, axis=0)
    w = np.zeros(d.shape[0])
    for (a, b), wt in zip(np.asarray(steps).reshape(-1, 2), weights):
        w[(d[:, 0] == a) & (d[:, 1] == b)] = wt
    if np.any(w == 0):
        return float("nan")  # a step outside the step set
    total = c[0] + float(np.sum(c[1:] * w))
    length = (wp[-1, 0] + wp[-1, 1]) - (wp[0, 0] + wp[0, 1])
    return total / length if length > 0 else float("nan")


def compare_results(pairs, best32, paths32, best64, paths64, steps, weights,
                    found32=None, found64=None):
    """Accumulated-cost error, path agreement and near-tie gaps."""
    n = len(pairs)
    rel, agree, gaps, gaps_own = [], 0, [], []
    for i in range(n):
        if found32 is not None and (not found32[i] or not found64[i]):
            continue
        b32, b64 = float(best32[i]), float(best64[i])
        rel.append(abs(b32 - b64) / max(abs(b64), 1e-300))
        same = paths32[i].shape == paths64[i].shape and np.array_equal(paths32[i], paths64[i])
        if same:
            agree += 1
            continue
        F1, F2 = pairs[i]
        s32 = path_score(F1, F2, paths32[i], steps, weights)
        s64 = path_score(F1, F2, paths64[i], steps, weights)
        gaps.append((s32 - b64) / abs(b64))
        gaps_own.append((s64 - b64) / abs(b64))
    rel = np.asarray(rel)
    out = {
        "pairs": int(len(rel)),
        "path_agreement_rate": agree / max(len(rel), 1),
        "divergent_pairs": int(len(gaps)),
        "best_cost_rel_err_max": float(rel.max()) if rel.size else None,
        "best_cost_rel_err_mean": float(rel.mean()) if rel.size else None,
    }
    if gaps:
        g = np.asarray(gaps)
        go = np.asarray(gaps_own)
        out.update({
            "divergent_fp32_path_fp64_score_rel_gap_max": float(np.nanmax(g)),
            "divergent_fp32_path_fp64_score_rel_gap_mean": float(np.nanmean(g)),
            "divergent_fp64_path_rescore_rel_dev_max": float(np.nanmax(np.abs(go))),
        })
    return out


def cost_error(plan32, plan64):
    """max / mean |C_fp32 - C_fp64| over one pair's cells (both plans loaded
    with the same features and tile length; cells outside tiles are 0 in
    both slabs and are left out of the mean)."""
    import torch
    a = plan32.view("COST").to(torch.float64)
    b = plan64.view("COST")
    valid = (a != 0) | (b != 0)
    d = (a - b).abs()
    return float(d.max().item()), float(d[valid].sum().item()), int(valid.sum().item())
