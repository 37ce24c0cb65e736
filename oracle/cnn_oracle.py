"""CPU restatement (numpy, FP64) of the tile proposer's kernels.

TEST INFRASTRUCTURE ONLY: tests/ compare the device kernels of
parflexdtw_b200/csrc/cnn.cu with these functions (forward values and
gradients); the product never calls them.  The proposer has no counterpart
in the reference, so these follow the kernels' own documented definitions
(include/parflexdtw_b200.h: pfx_pool_features ... pfx_tile_mask_from_scores).
"""
from __future__ import annotations

import numpy as np


def pool_features(F, pool):
    """(d, n) -> (d, ceil(n / pool)): block means of the L2-normalised frames."""
    F = np.asarray(F, dtype=np.float64)
    A = F / np.sqrt(np.sum(F * F, axis=0, keepdims=True))
    d, n = A.shape
    P = -(-n // pool)
    out = np.zeros((d, P))
    for p in range(P):
        out[:, p] = A[:, p * pool:min(n, (p + 1) * pool)].mean(axis=1)
    return out


def pooled_cost(A, B):
    return 1.0 - np.asarray(A, np.float64).T @ np.asarray(B, np.float64)


def center(P):
    P = np.asarray(P, np.float64)
    X = P - P.mean(axis=1, keepdims=True) - P.mean(axis=0, keepdims=True) + P.mean()
    return X / np.sqrt(np.mean(X * X))


def _taps(xp, ky, kx, stride, Ho, Wo):
    return xp[:, ky:ky + stride * (Ho - 1) + 1:stride, kx:kx + stride * (Wo - 1) + 1:stride]


def conv3x3(x, w, b, stride, relu):
    """x (Cin, H, W), w (Cout, Cin, 3, 3), zero padding 1 -> (Cout, Ho, Wo)."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    Cin, H, W = x.shape
    Ho, Wo = (H - 1) // stride + 1, (W - 1) // stride + 1
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1)))
    out = np.zeros((w.shape[0], Ho, Wo))
    for ky in range(3):
        for kx in range(3):
            out += np.einsum("oc,chw->ohw", w[:, :, ky, kx], _taps(xp, ky, kx, stride, Ho, Wo))
    out += np.asarray(b, np.float64)[:, None, None]
    return np.maximum(out, 0.0) if relu else out


def conv3x3_backward(x, w, stride, y, relu, dy):
    """Gradients (dx, dw, db) of conv3x3 for the gradient dy at its output y."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    dy = np.asarray(dy, np.float64)
    dz = dy * (np.asarray(y) > 0) if relu else dy
    Cin, H, W = x.shape
    Ho, Wo = dz.shape[1:]
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1)))
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for ky in range(3):
        for kx in range(3):
            dw[:, :, ky, kx] = np.einsum("ohw,chw->oc", dz, _taps(xp, ky, kx, stride, Ho, Wo))
            dxp[:, ky:ky + stride * (Ho - 1) + 1:stride, kx:kx + stride * (Wo - 1) + 1:stride] += \
                np.einsum("oc,ohw->chw", w[:, :, ky, kx], dz)
    return dxp[:, 1:-1, 1:-1], dw, dz.sum(axis=(1, 2))


def tile_regions(H, W, n1, n2, hop, L, N, M, fpp):
    """Per tile: (y0, y1, x0, x1) of its region of the logit map."""
    out = []
    for t in range(n1 * n2):
        i, j = divmod(t, n2)
        r0, c0 = i * hop, j * hop
        r1, c1 = min(N, r0 + L), min(M, c0 + L)
        y0, y1 = min(r0 // fpp, H - 1), min(-(-r1 // fpp), H)
        x0, x1 = min(c0 // fpp, W - 1), min(-(-c1 // fpp), W)
        out.append((y0, max(y1, y0 + 1), x0, max(x1, x0 + 1)))
    return out


def tile_max(logits, n1, n2, hop, L, N, M, fpp):
    H, W = logits.shape
    score = np.zeros(n1 * n2)
    arg = np.zeros(n1 * n2, np.int64)
    for t, (y0, y1, x0, x1) in enumerate(tile_regions(H, W, n1, n2, hop, L, N, M, fpp)):
        reg = logits[y0:y1, x0:x1]
        k = int(np.argmax(reg))  # first (lowest flat index) maximum
        yy, xx = divmod(k, reg.shape[1])
        score[t] = reg[yy, xx]
        arg[t] = (y0 + yy) * W + x0 + xx
    return score, arg


def bce(score, label, pos_weight):
    s = np.asarray(score, np.float64)
    y = np.asarray(label, np.float64)
    wt = np.where(y > 0, pos_weight, 1.0)
    n = s.size
    loss = np.sum(wt * (np.log1p(np.exp(-np.abs(s))) + np.maximum(s, 0) - s * y)) / n
    return loss, wt * (1.0 / (1.0 + np.exp(-s)) - y) / n
