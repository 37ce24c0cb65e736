"""Seeded synthetic chroma-like sequence pairs for tests and benchmarks.

The reference's own evaluation data (audio chroma of piano recordings) is not
available, so every workload here is generated: non-negative 12-d frames drawn
from a Dirichlet(0.3) distribution (chroma vectors are sparse and
non-negative), L2-normalised per frame; the second sequence is the first one
resampled along a random monotone piecewise-linear time warp plus noise, and
optionally padded with unrelated frames at both ends so that FlexDTW's free
start / free end matter.

Feature layout follows the reference: ``F`` has shape ``(d, frames)`` and the
cost matrix is ``C = 1 - L2norm(F1).T @ L2norm(F2)`` with shape ``(N, M)``
(``FlexDTW.py:213-216``, ``Parflex.py:1470``).
"""
from __future__ import annotations

import numpy as np

__all__ = [
    "l2norm",
    "cost_matrix_host",
    "cost_matrix_det",
    "chroma_sequence",
    "warped_pair",
    "PairSpec",
    "CONFIG0",
    "CONFIG1",
    "NCU_SMALL",
    "WORKLOADS",
    "make_pair",
]


def l2norm(F: np.ndarray) -> np.ndarray:
    """Column L2 normalisation with the reference's ``+1e-9`` on the norm
    (``FlexDTW.py:213-216``)."""
    n = np.sqrt(np.sum(F * F, axis=0)) + 1e-9
    return F / n.reshape((1, -1))


def cost_matrix_host(F1: np.ndarray, F2: np.ndarray) -> np.ndarray:
    """Host FP64 cosine cost exactly as the reference builds it
    (``Parflex.py:1470``)."""
    return 1 - l2norm(F1).T @ l2norm(F2)


def cost_matrix_det(F1: np.ndarray, F2: np.ndarray) -> np.ndarray:
    """FP64 cosine cost with a fixed summation order (k = 0, 1, ..., d-1).

    Each product and each running sum is one IEEE-rounded numpy ufunc, so the
    result is bit-identical on every machine (a BLAS GEMM's blocking and FMA
    use are not).  Golden fixtures and parity tests feed this same ``C`` to the
    reference and to the device path.
    """
    A = l2norm(np.asarray(F1, dtype=np.float64))
    B = l2norm(np.asarray(F2, dtype=np.float64))
    acc = A[0][:, None] * B[0][None, :]
    for k in range(1, A.shape[0]):
        acc = acc + A[k][:, None] * B[k][None, :]
    return 1.0 - acc


def chroma_sequence(rng: np.random.Generator, n: int, d: int = 12,
                    alpha: float = 0.3) -> np.ndarray:
    """``n`` Dirichlet(alpha) frames of dimension ``d``, L2-normalised, (d, n)."""
    F = rng.dirichlet(np.full(d, alpha), size=n).T
    return l2norm(F)


def _warp_positions(rng: np.random.Generator, n_src: int, m_target: int,
                    seg_lo: int = 40, seg_hi: int = 200,
                    slope_lo: float = 0.7, slope_hi: float = 1.4) -> np.ndarray:
    """Monotone piecewise-linear map from ``m_target`` output frames to
    fractional source positions in ``[0, n_src-1]``.

    Segment lengths (in source frames) are U(seg_lo, seg_hi); each segment's
    local tempo ratio (output frames per source frame) is U(slope_lo, slope_hi),
    then all ratios are scaled by one common factor so the total output length
    is ``m_target``.
    """
    lens, slopes = [], []
    total = 0
    while total < n_src - 1:
        L = int(rng.integers(seg_lo, seg_hi + 1))
        L = min(L, n_src - 1 - total)
        lens.append(L)
        slopes.append(rng.uniform(slope_lo, slope_hi))
        total += L
    lens = np.asarray(lens, dtype=np.float64)
    slopes = np.asarray(slopes, dtype=np.float64)
    out_lens = lens * slopes
    out_lens *= (m_target - 1) / out_lens.sum()
    # knots: output position -> source position
    out_knots = np.concatenate([[0.0], np.cumsum(out_lens)])
    src_knots = np.concatenate([[0.0], np.cumsum(lens)])
    m = np.arange(m_target, dtype=np.float64)
    return np.interp(m, out_knots, src_knots)


def warped_pair(rng: np.random.Generator, n: int, m_core: int, d: int = 12,
                noise: float = 0.05, pad_frac: float = 0.0,
                latent: str = "dirichlet"):
    """One (F1, F2) pair.

    ``F1``: ``n`` frames.  ``F2``: ``F1`` resampled (linear interpolation) at
    the warp positions (``m_core`` frames), plus N(0, noise) noise, clipped at
    0 for chroma (non-negative) latents, renormalised; then, when
    ``pad_frac > 0``, U(0, pad_frac) * m_core unrelated frames are prepended
    and appended.
    """
    if latent == "dirichlet":
        F1 = chroma_sequence(rng, n, d)
    else:
        F1 = l2norm(rng.standard_normal((d, n)))
    pos = _warp_positions(rng, n, m_core)
    i0 = np.floor(pos).astype(np.int64)
    i1 = np.minimum(i0 + 1, n - 1)
    t = (pos - i0)[None, :]
    F2 = F1[:, i0] * (1.0 - t) + F1[:, i1] * t
    F2 = F2 + rng.normal(0.0, noise, size=F2.shape)
    if latent == "dirichlet":
        F2 = np.clip(F2, 0.0, None)
    F2 = l2norm(F2)
    if pad_frac > 0:
        pre = int(rng.uniform(0, pad_frac) * m_core)
        post = int(rng.uniform(0, pad_frac) * m_core)
        parts = []
        if pre:
            parts.append(chroma_sequence(rng, pre, d) if latent == "dirichlet"
                         else l2norm(rng.standard_normal((d, pre))))
        parts.append(F2)
        if post:
            parts.append(chroma_sequence(rng, post, d) if latent == "dirichlet"
                         else l2norm(rng.standard_normal((d, post))))
        F2 = np.concatenate(parts, axis=1)
    return np.ascontiguousarray(F1), np.ascontiguousarray(F2)


class PairSpec:
    """Named workload: sizes, tile length and DP parameters."""

    def __init__(self, name, n, m_core, L, pad_frac=0.0, d=12, noise=0.05,
                 weights=(2.0, 3.0, 3.0), beta=0.1, seed=0):
        self.name = name
        self.n = n
        self.m_core = m_core
        self.L = L
        self.pad_frac = pad_frac
        self.d = d
        self.noise = noise
        self.steps = ((1, 1), (1, 2), (2, 1))
        self.weights = tuple(float(w) for w in weights)
        self.beta = beta
        self.seed = seed

    def describe(self):
        return {"workload": self.name, "N": self.n, "M_core": self.m_core,
                "L": self.L, "pad_frac": self.pad_frac, "d": self.d,
                "weights": list(self.weights), "beta": self.beta,
                "seed": self.seed}


# One pair, 2000 x ~2400 frames, L=500 (runs on CPU in well under a second).
CONFIG0 = PairSpec("chroma12_pair_2000x2400_L500", 2000, 2400, 500)
# One long pair, 30000 x ~36000 frames (+0-10 % unrelated padding per end),
# L=4000, FP64 DP.
CONFIG1 = PairSpec("chroma12_pair_30000x36000_L4000_fp64", 30000, 36000, 4000,
                   pad_frac=0.10)
# Profiling case: the 30000 x 36000 workload's tile length and kernel
# configuration on a 3 x 3 tile grid (C = 0.6 GB, larger than L2).
NCU_SMALL = PairSpec("chroma12_pair_8000x9600_L4000_fp64", 8000, 9600, 4000,
                     pad_frac=0.0)



class BatchSpec:
    """Named batch workload: ``n_pairs`` pairs with N ~ U(n_lo, n_hi) and
    M = N x U(ratio_lo, ratio_hi) through the warp model of ``warped_pair``;
    tile length per pair from ``L_choices`` (the autotuner picks per length
    bucket when more than one is given)."""

    def __init__(self, name, n_pairs, n_lo, n_hi, ratio_lo=0.7, ratio_hi=1.4,
                 L_choices=(1000, 2000), pad_frac=0.0, d=12, noise=0.05,
                 weights=(2.0, 3.0, 3.0), beta=0.1, seed=0):
        self.name = name
        self.n_pairs = n_pairs
        self.n_lo, self.n_hi = n_lo, n_hi
        self.ratio_lo, self.ratio_hi = ratio_lo, ratio_hi
        self.L_choices = tuple(int(x) for x in L_choices)
        self.pad_frac = pad_frac
        self.d = d
        self.noise = noise
        self.steps = ((1, 1), (1, 2), (2, 1))
        self.weights = tuple(float(w) for w in weights)
        self.beta = beta
        self.seed = seed

    def describe(self):
        return {"workload": self.name, "pairs": self.n_pairs,
                "N_range": [self.n_lo, self.n_hi],
                "M_over_N": [self.ratio_lo, self.ratio_hi],
                "L_choices": list(self.L_choices), "d": self.d,
                "weights": list(self.weights), "beta": self.beta, "seed": self.seed}


def make_batch(spec: BatchSpec, seed_offset: int = 0):
    """Generate the ``n_pairs`` (F1, F2) pairs of a batch spec."""
    rng = np.random.default_rng(spec.seed + seed_offset)
    out = []
    for _ in range(spec.n_pairs):
        n = int(rng.integers(spec.n_lo, spec.n_hi + 1))
        m = int(round(n * rng.uniform(spec.ratio_lo, spec.ratio_hi)))
        out.append(warped_pair(rng, n, m, d=spec.d, noise=spec.noise,
                               pad_frac=spec.pad_frac))
    return out


# 256 pairs, N ~ U(2000, 20000), M = N x U(0.7, 1.4), 12-d chroma-like
# features, L in {1000, 2000} per length bucket, FP64 DP.
BATCH256 = BatchSpec("chroma12_batch256_N2000-20000_fp64", 256, 2000, 20000)



class PrecisionSpec:
    """Named precision workload: ``n_pairs`` pairs with N, M ~ U(lo, hi)
    independently; each pair from one ``d``-dimensional Gaussian latent
    sequence (F1 = its L2-normalised frames, F2 = F1 under the warp model
    plus N(0, noise) noise, re-normalised); one tile length ``L``."""

    def __init__(self, name, n_pairs, lo, hi, d=128, noise=0.1, L=1000,
                 weights=(2.0, 3.0, 3.0), beta=0.1, seed=0):
        self.name = name
        self.n_pairs = n_pairs
        self.lo, self.hi = lo, hi
        self.d = d
        self.noise = noise
        self.L = L
        self.steps = ((1, 1), (1, 2), (2, 1))
        self.weights = tuple(float(w) for w in weights)
        self.beta = beta
        self.seed = seed

    def describe(self):
        return {"workload": self.name, "pairs": self.n_pairs, "N_range": [self.lo, self.hi],
                "M_range": [self.lo, self.hi], "d": self.d, "latent": "gaussian",
                "noise": self.noise, "L": self.L, "weights": list(self.weights),
                "beta": self.beta, "seed": self.seed}


def make_precision_batch(spec: PrecisionSpec, seed_offset: int = 0, n_pairs=None):
    """Generate the (F1, F2) pairs of a precision spec (the first ``n_pairs``)."""
    rng = np.random.default_rng(spec.seed + seed_offset)
    out = []
    for _ in range(spec.n_pairs if n_pairs is None else n_pairs):
        n = int(rng.integers(spec.lo, spec.hi + 1))
        m = int(rng.integers(spec.lo, spec.hi + 1))
        out.append(warped_pair(rng, n, m, d=spec.d, noise=spec.noise, latent="gaussian"))
    return out


# 2048 pairs, N, M ~ U(1000, 8000), 128-d Gaussian latents, L = 1000: the FP32
# form (bf16 tensor-core cost, FP32 DP) against the FP64 plain form.
PRECISION2048 = PrecisionSpec("gauss128_batch2048_N1000-8000_L1000_fp32_vs_fp64", 2048,
                              1000, 8000)



class PruneSpec(BatchSpec):
    """Named learned-pruning workload: long pairs aligned one at a time with
    the full-tile FP64 method and with the tile proposer."""


# 64 pairs, N ~ U(40000, 60000), M = N x U(0.7, 1.4), 12-d chroma-like
# features with 0-10 % unrelated padding per end, L = 2000.
PRUNE64 = PruneSpec("chroma12_pairs64_N40000-60000_L2000_pruned", 64, 40000, 60000,
                    L_choices=(2000,), pad_frac=0.10)

# Profiling case of the same method: 4 pairs, N ~ U(8000, 10000) (about 3 GB
# of cost slabs on the device), L = 2000.
PRUNE_NCU = PruneSpec("chroma12_pairs4_N8000-10000_L2000_pruned", 4, 8000, 10000,
                      L_choices=(2000,), pad_frac=0.10)

# Profiling case of the stage-1 kernel as the learned-pruning workload runs it
# (4 warps per tile CTA, four CTAs per SM: 720 tiles of up to 1000 x 1000,
# about 6 GB of cost slabs): 20 pairs, N ~ U(5000, 6000), L = 1000.
PRUNE_NCU_W4 = PruneSpec("chroma12_pairs20_N5000-6000_L1000_pruned", 20, 5000, 6000,
                         L_choices=(1000,), pad_frac=0.10)

# Per-cell counters of the stage-1 kernel at the learned-pruning workload's
# tile length (L = 2000, run with --warps 4 for its kernel variant): 4 pairs,
# N ~ U(10000, 12000), about 5 GB of cost slabs.
PRUNE_NCU_L2000 = PruneSpec("chroma12_pairs4_N10000-12000_L2000_pruned", 4, 10000, 12000,
                            L_choices=(2000,), pad_frac=0.10)


class ShardSpec(PairSpec):
    """Named one-pair workload whose tiles are sharded across ranks."""


# One square pair of 100000 x 100000 frames at L = 4000: 26 x 26 = 676 tiles,
# 1.0e10 DP cells, far more tiles than one GPU has SMs; its tiles split
# across ranks (one edge exchange), or all on one GPU (89 GB of FP64 cost).
SHARD1 = ShardSpec("chroma12_pair_100000x100000_L4000_tile_sharded", 100000, 100000, 4000)

# Small cases of the batch, precision and sharded-pair workloads (seconds per
# run): every arm of the benchmark is exercised end to end by the tests.
BATCH_SMALL = BatchSpec("chroma12_batch12_N2000-6000_fp64", 12, 2000, 6000)
PRECISION_SMALL = PrecisionSpec("gauss128_batch24_N1000-3000_L1000_fp32_vs_fp64", 24,
                                1000, 3000)
SHARD_SMALL = ShardSpec("chroma12_pair_12000x12000_L2000_tile_sharded", 12000, 12000, 2000)

WORKLOADS = {"config0": CONFIG0, "config1": CONFIG1, "ncu_small": NCU_SMALL,
             "batch256": BATCH256, "precision2048": PRECISION2048, "prune64": PRUNE64,
             "prune_ncu": PRUNE_NCU, "prune_ncu_w4": PRUNE_NCU_W4,
             "prune_ncu_l2000": PRUNE_NCU_L2000,
             "shard1": SHARD1, "batch_small": BATCH_SMALL,
             "precision_small": PRECISION_SMALL, "shard_small": SHARD_SMALL}


def make_pair(spec: PairSpec):
    """Generate ``(F1, F2)`` for a spec from its seed."""
    rng = np.random.default_rng(spec.seed)
    return warped_pair(rng, spec.n, spec.m_core, d=spec.d, noise=spec.noise,
                       pad_frac=spec.pad_frac)
