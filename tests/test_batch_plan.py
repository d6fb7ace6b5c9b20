"""Host-side work decomposition of batches (no GPU): the library's plan
against a restatement of its rules, and the coverage invariants the kernel
relies on (every unit owned by exactly one CTA pair, partial slots enough)."""
import numpy as np
import pytest

import matching_sift_b200 as ms

BN = 128


def _restated(pairs, qpt, workers):
    group = 2 * qpt * 128
    units = tiles = queries = 0
    groups = []
    for na, nb, _ in pairs:
        g = -(-na // group)
        t = -(-nb // BN)
        for k in range(g if t else 0):
            groups.append((units + k * t, t))
        units += g * t
        tiles += t
        queries += na
    grid = min(workers, units)
    w0 = lambda c: (c * units) // grid
    cta_of = lambda w: ((w + 1) * grid - 1) // units
    ms_ = 1
    for first, t in groups:
        ms_ = max(ms_, cta_of(first + t - 1) - cta_of(first) + 1)
    return units, tiles, queries, (ms_ if grid else 1), grid, group, w0, cta_of


@pytest.mark.parametrize("qpt", [1, 2])
@pytest.mark.parametrize("workers", [1, 7, 74])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_batch_decomposition_matches_restatement(qpt, workers, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 60))
    na = np.exp(rng.uniform(0, np.log(9000), n)).astype(int)
    nb = np.exp(rng.uniform(0, np.log(9000), n)).astype(int)
    na[rng.random(n) < 0.1] = 0
    nb[rng.random(n) < 0.1] = 0
    offs = np.concatenate([[0], np.cumsum(nb)[:-1]])
    pairs = np.stack([na, nb, offs], 1)
    got = ms.batch_describe(pairs, int(nb.sum()), qpt=qpt, workers=workers)
    units, tiles, queries, max_splits, grid, group, w0, cta_of = _restated(pairs.tolist(), qpt, workers)
    assert (got["units"], got["tiles"], got["queries"], got["grid"], got["group_rows"]) == \
        (units, tiles, queries, grid, group)
    assert got["max_splits"] == max_splits
    if grid:
        # contiguous ranges cover every unit once, and cta_of inverts w0
        owners = np.concatenate([np.full(w0(c + 1) - w0(c), c) for c in range(grid)])
        assert len(owners) == units
        assert all(cta_of(w) == owners[w] for w in range(0, units, max(1, units // 500)))


def test_batch_describe_rejects_out_of_range_base():
    with pytest.raises(ms.SiftError):
        ms.batch_describe([[10, 5, 3]], 7)
    with pytest.raises(ms.SiftError):
        ms.batch_describe([[10, 5, 0]], 7, qpt=3)
