"""Host logic of learned pruning (no GPU): the test that decides whether a
pruned run's path came near a pruned tile, against a brute-force statement
of the same rule."""
import numpy as np
import pytest

pytest.importorskip("torch")
from parflexdtw_b200.prune import _needs_fallback, _pruned_near_path, tiles_on_path  # noqa: E402


def _brute(wp, mask, N, M, L, B):
    """Pruned tiles covering a cell of the 3 x 3 block neighbourhood (B x B
    blocks) of a block the path touches."""
    n1, n2 = mask.shape
    hop = L - 1
    near = np.zeros_like(mask, bool)
    for rb, cb in {(int(r) // B, int(c) // B) for r, c in wp}:
        r0, r1 = max(rb - 1, 0) * B, min((rb + 2) * B, N) - 1
        c0, c1 = max(cb - 1, 0) * B, min((cb + 2) * B, M) - 1
        for i in range(n1):
            if not (i * hop <= r1 and i * hop + L - 1 >= r0):
                continue
            for j in range(n2):
                if j * hop <= c1 and j * hop + L - 1 >= c0 and not mask[i, j]:
                    near[i, j] = True
    return near


def _path(rng, N, M):
    r, c = [0], [0]
    while r[-1] < N - 1 or c[-1] < M - 1:
        k = rng.integers(3)
        dr, dc = [(1, 1), (1, 2), (2, 1)][k]
        r.append(min(r[-1] + dr, N - 1))
        c.append(min(c[-1] + dc, M - 1))
    return np.stack([r, c], axis=1)


@pytest.mark.parametrize("seed", range(6))
def test_pruned_near_path_matches_brute_force(seed):
    rng = np.random.default_rng(seed)
    N, M, L, B = int(rng.integers(300, 900)), int(rng.integers(300, 900)), 100, 16
    wp = _path(rng, N, M)
    hop = L - 1
    n1, n2 = -(-(N - 1) // hop), -(-(M - 1) // hop)
    on = tiles_on_path(wp, N, M, L).astype(bool)
    for keep in (0.0, 0.5, 0.9):
        mask = on | (rng.random((n1, n2)) < keep)
        got = _pruned_near_path(wp, mask, N, M, L, B)
        want = _brute(wp, mask, N, M, L, B)
        assert np.array_equal(got, want)
        assert _needs_fallback(wp, mask, N, M, L, B) == bool(want.any())
    assert not _pruned_near_path(wp, np.ones((n1, n2), bool), N, M, L, B).any()
