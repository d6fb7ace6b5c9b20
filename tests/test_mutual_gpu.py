"""Mutual nearest neighbours (cross-check) of image pairs through the C ABI,
against the oracle composed of exact 2-NN in both directions."""
import numpy as np
import pytest

import matching_sift_b200 as ms
import oracle
from matching_sift_b200 import datagen

pytestmark = pytest.mark.gpu


def _pairs(seed, n_pairs, contiguous):
    """First sets a (concatenated), second sets b and pair rows {n_a, n_b, b_off}:
    second sets are 40% noisy copies of the first (so most rows have a
    mutual partner); with contiguous=False they are stored in reverse order
    and one pair reuses another's set (the gather path)."""
    rng = np.random.default_rng([seed, 5])
    sizes = [(int(x), int(y)) for x, y in np.exp(rng.uniform(np.log(20), np.log(1500), (n_pairs, 2))).astype(int)]
    sizes += [(0, 40), (30, 0), (1, 1), (129, 2)]
    firsts, seconds = [], []
    for k, (na, nb) in enumerate(sizes):
        a = datagen.make_base(na, seed=seed * 100 + k)
        if na and nb:
            nc = min(int(0.4 * nb), na)
            b = np.concatenate([datagen.make_queries(nc, a, seed=seed * 100 + k, copy_frac=1.0),
                                datagen.make_base(nb - nc, seed=seed * 100 + k + 50)])
        else:
            b = datagen.make_base(nb, seed=seed * 100 + k + 50)
        firsts.append(a)
        seconds.append(b)
    order = range(len(sizes)) if contiguous else reversed(range(len(sizes)))
    offs, rows, chunks = {}, 0, []
    for k in order:
        offs[k] = rows
        rows += seconds[k].shape[0]
        chunks.append(seconds[k])
    b_all = np.concatenate(chunks)
    pairs = [[sizes[k][0], sizes[k][1], offs[k]] for k in range(len(sizes))]
    a_all = np.concatenate(firsts)
    if not contiguous:  # one more pair searching against pair 0's second set
        extra = datagen.make_queries(70, seconds[0], seed=seed + 7, copy_frac=0.6)
        a_all = np.concatenate([a_all, extra])
        firsts.append(extra)
        pairs.append([70, sizes[0][1], offs[0]])
    return a_all, b_all, np.array(pairs, np.uint32), firsts


def _check(a, b, pairs, out, threshold):
    m = out["matches"].cpu().numpy().view(np.uint32)
    idx = out["nn_idx"].cpu().numpy()
    row = 0
    mutual = 0
    for na, nb, off in pairs:
        na, nb, off = int(na), int(nb), int(off)
        sl = slice(row, row + na)
        row += na
        want = oracle.mutual_match(a[sl], b[off:off + nb], threshold)
        np.testing.assert_array_equal(m[sl], want, err_msg=f"pair {na}x{nb}@{off}")
        _, i = oracle.brute_2nn_u8(a[sl], b[off:off + nb])
        np.testing.assert_array_equal(idx[sl], i)
        mutual += int((want != 0xFFFFFFFF).sum())
    assert mutual > 0


def _dev(x, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x)).to(dev)


@pytest.mark.parametrize("contiguous", [True, False])
@pytest.mark.parametrize("threshold", [0.0, 0.8])
def test_mutual_batch_vs_oracle(cuda_device, contiguous, threshold):
    a, b, pairs, _ = _pairs(3 if contiguous else 4, 20, contiguous)
    out = ms.match_mutual_batch(_dev(a, cuda_device), _dev(b, cuda_device), pairs, threshold)
    assert ms.stream_status() == ms.SIFT_OK
    _check(a, b, pairs, out, threshold)


def test_mutual_single_pair_is_symmetric(cuda_device):
    a = datagen.make_base(900, seed=11)
    b = datagen.make_queries(700, a, seed=12, copy_frac=0.7)
    ad, bd = _dev(a, cuda_device), _dev(b, cuda_device)
    ab = ms.match_mutual(ad, bd, threshold=0.0)["matches"].cpu().numpy().view(np.uint32)
    ba = ms.match_mutual(bd, ad, threshold=0.0)["matches"].cpu().numpy().view(np.uint32)
    np.testing.assert_array_equal(ab, oracle.mutual_match(a, b, 0.0))
    # without the ratio test the relation is symmetric
    pairs_ab = {(i, int(j)) for i, j in enumerate(ab) if j != 0xFFFFFFFF}
    pairs_ba = {(int(j), i) for i, j in enumerate(ba) if j != 0xFFFFFFFF}
    assert pairs_ab == pairs_ba and len(pairs_ab) > 300


def _expected_lists(m, dist, pairs):
    recs, offs, row = [], [], 0
    for p, (na, nb, off) in enumerate(pairs):
        offs.append(len(recs))
        for a in range(int(na)):
            j = m[row + a]
            if j != 0xFFFFFFFF:
                recs.append((p, a, int(j), dist[row + a, 0], dist[row + a, 1]))
        row += int(na)
    offs.append(len(recs))
    return recs, offs


@pytest.mark.parametrize("contiguous", [True, False])
def test_match_lists_for_verification(cuda_device, contiguous):
    """Compaction of mutual matches into per-pair lists equals a row-order
    filter of the same outputs (grouped by pair, offsets, distances)."""
    a, b, pairs, _ = _pairs(6 if contiguous else 7, 30, contiguous)
    out = ms.match_mutual_batch(_dev(a, cuda_device), _dev(b, cuda_device), pairs, 0.8)
    lists = ms.compact_matches(out, pairs)
    assert ms.stream_status() == ms.SIFT_OK
    m = out["matches"].cpu().numpy().view(np.uint32)
    dist = out["nn_dist"].cpu().numpy()
    recs, offs = _expected_lists(m, dist, pairs)
    assert len(recs) > 100
    np.testing.assert_array_equal(lists["offsets"].cpu().numpy(), offs)
    got = np.stack([lists[k].cpu().numpy().astype(np.float64) for k in ("pair", "a", "b", "d1", "d2")], 1)
    np.testing.assert_array_equal(got, np.array(recs, np.float64))
    # a capacity below the count: the first `capacity` records, the full count in the offsets
    cap = len(recs) // 3
    part = ms.compact_matches(out, pairs, capacity=cap)
    assert int(part["offsets"][-1]) == len(recs) and part["a"].shape[0] == cap
    np.testing.assert_array_equal(part["b"].cpu().numpy(), got[:cap, 2])


def test_match_lists_of_a_plain_batch(cuda_device):
    """Lists from the one-shot batch (ratio-test matches) and without distances."""
    a, b, pairs, _ = _pairs(8, 12, True)
    out = ms.match_batch(_dev(a, cuda_device), _dev(b, cuda_device), pairs, 0.8)
    m = out["matches"].cpu().numpy().view(np.uint32)
    lists = ms.compact_matches({"matches": out["matches"]}, pairs)
    recs, offs = _expected_lists(m, np.zeros((m.shape[0], 2), np.float32), pairs)
    np.testing.assert_array_equal(lists["offsets"].cpu().numpy(), offs)
    np.testing.assert_array_equal(lists["a"].cpu().numpy(), [r[1] for r in recs])
    assert (lists["d1"].cpu().numpy() == 0).all()
