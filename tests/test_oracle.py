"""The CPU oracle is pinned against the reference's own outputs (no GPU needed)."""
import glob
import os

import numpy as np
import pytest

import oracle
from matching_sift_b200 import datagen

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FLT_MAX = np.float32(np.finfo(np.float32).max)


def _golden(prefix):
    files = sorted(glob.glob(os.path.join(GOLDEN, prefix + "*.npz")))
    assert files, f"no {prefix} fixtures"
    return files


@pytest.mark.parametrize("path", _golden("host_brute_"), ids=os.path.basename)
def test_oracle_reproduces_reference_host_brute(path):
    """host_brute (src/knn_brute.cu:801) output == the C restatement, bit for bit."""
    z = np.load(path)
    q, r, ref = z["q"], z["r"], z["sorted"]
    d, i = oracle.brute_2nn_u8(q, r)
    present1 = i[:, 0] >= 0
    present2 = i[:, 1] >= 0
    assert present1.all()
    np.testing.assert_array_equal(ref[:, 2].astype(np.int64), i[:, 0])
    np.testing.assert_array_equal(ref[:, 0].astype(np.int64), d[:, 0])
    np.testing.assert_array_equal(ref[present2, 3].astype(np.int64), i[present2, 1])
    np.testing.assert_array_equal(ref[present2, 1].astype(np.int64), d[present2, 1])
    # absent second neighbour: the reference leaves MAXFLOAT in both fields
    assert (ref[~present2, 1] == FLT_MAX).all() and (ref[~present2, 3] == FLT_MAX).all()


def test_oracle_vs_live_reference():
    if not oracle.ref_available():
        pytest.skip("reference library not built here")
    q, r = datagen.make_workload(64, 3000, seed=99)
    ref = oracle.ref_host_brute(q.astype(np.float32), r.astype(np.float32), nthreads=4)
    d, i = oracle.brute_2nn_u8(q, r)
    np.testing.assert_array_equal(ref[:, 2].astype(np.int64), i[:, 0])
    np.testing.assert_array_equal(ref[:, 3].astype(np.int64), i[:, 1])
    np.testing.assert_array_equal(ref[:, :2].astype(np.int64), d)


def test_dot_metric_matches_numpy():
    q, r = datagen.make_workload(40, 500, seed=3)
    d, i = oracle.brute_2nn_u8(q, r, metric=1)
    key = -2 * (q.astype(np.int64) @ r.astype(np.int64).T)
    order = np.lexsort((np.broadcast_to(np.arange(r.shape[0]), key.shape), key), axis=1)
    np.testing.assert_array_equal(order[:, :2], i)
    np.testing.assert_array_equal(np.take_along_axis(key, order[:, :2], 1), d)


def test_l2_matches_numpy_lexicographic():
    q, r = datagen.make_workload(50, 700, seed=4)
    r[10] = r[20]  # a duplicate pair creates exact ties
    q[0] = r[20]
    d, i = oracle.brute_2nn_u8(q, r)
    full = ((q[:, None, :].astype(np.int64) - r[None, :, :].astype(np.int64)) ** 2).sum(-1)
    order = np.lexsort((np.broadcast_to(np.arange(r.shape[0]), full.shape), full), axis=1)
    np.testing.assert_array_equal(order[:, :2], i)
    assert i[0, 0] == 10 and i[0, 1] == 20 and d[0, 0] == 0 and d[0, 1] == 0


def test_f64_oracle_agrees_with_integer_oracle():
    q, r = datagen.make_workload(30, 400, seed=8)
    d, i = oracle.brute_2nn_u8(q, r)
    df, jf = oracle.brute_2nn_f64(q.astype(np.float32), r.astype(np.float32))
    np.testing.assert_array_equal(i, jf)
    np.testing.assert_array_equal(d.astype(np.float64), df)


def test_ratio_match_semantics():
    dist = np.array([[100, 400], [100, 156], [0, 0], [50, np.iinfo(np.int64).max]], np.int64)
    idx = np.array([[7, 8], [9, 10], [11, 12], [13, -1]], np.int64)
    m = oracle.ratio_match(dist, idx, 0.8)
    # sqrt(100)/sqrt(400) = 0.5 < 0.8 ; sqrt(100)/sqrt(156) = 0.8006 >= 0.8 ; 0/0 = NaN fails ; no 2nd -> 0
    np.testing.assert_array_equal(m, np.array([7, 0xFFFFFFFF, 0xFFFFFFFF, 13], np.uint32))


def test_generator_is_seeded_and_shaped():
    a = datagen.make_base(300, seed=7)
    b = datagen.make_base(300, seed=7)
    c = datagen.make_base(300, seed=8)
    assert a.dtype == np.uint8 and a.shape == (300, 128)
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
    norms = np.sqrt((a.astype(np.float64) ** 2).sum(1))
    assert abs(norms.mean() - 512) < 3
    assert ((a == 0).sum(1) >= 38).all()
    q = datagen.make_queries(200, a, seed=7)
    # half of the queries are noisy copies: their nearest base row is close
    d, _ = oracle.brute_2nn_u8(q, a)
    assert (d[:, 0] < 20000).sum() >= 90


def test_bucket_sort_groups_by_code():
    rng = np.random.default_rng(0)
    code = rng.integers(0, 16, 1000).astype(np.uint32)
    order, bc, bs, bn = oracle.bucket_sort(code)
    assert bn.sum() == 1000 and (np.diff(bc.astype(np.int64)) > 0).all()
    for k in range(len(bc)):
        members = order[bs[k]:bs[k] + bn[k]]
        assert (code[members] == bc[k]).all() and (np.diff(members) > 0).all()
        np.testing.assert_array_equal(np.sort(np.nonzero(code == bc[k])[0]), members)


def test_lsh_scan_is_exact_on_candidates():
    q, r = datagen.make_workload(20, 300, seed=2)
    planes = datagen.make_hyperplanes(4, 2, seed=2)
    qc = np.stack([oracle.lsh_codes(q, planes[t])[0] for t in range(2)])
    rc = np.stack([oracle.lsh_codes(r, planes[t])[0] for t in range(2)])
    d, i = oracle.lsh_scan(q, r, qc, rc)
    for k in range(q.shape[0]):
        cand = np.nonzero((rc[0] == qc[0, k]) | (rc[1] == qc[1, k]))[0]
        if cand.size == 0:
            assert i[k, 0] == -1
            continue
        dd = ((r[cand].astype(np.int64) - q[k].astype(np.int64)) ** 2).sum(1)
        o = np.lexsort((cand, dd))
        assert i[k, 0] == cand[o[0]] and d[k, 0] == dd[o[0]]
        if cand.size > 1:
            assert i[k, 1] == cand[o[1]] and d[k, 1] == dd[o[1]]


def test_mutual_oracle_small_example():
    """Mutual nearest neighbours on hand-made sets: rows 0 and 1 of a pick
    each other's partners in b; row 2 of a prefers b[0], which prefers a[0]."""
    a = np.zeros((3, 128), np.uint8)
    b = np.zeros((2, 128), np.uint8)
    a[0, 0], a[1, 1], a[2, 0], a[2, 2] = 100, 100, 90, 30
    b[0, 0], b[1, 1] = 101, 99
    m = oracle.mutual_match(a, b, 0.0)
    assert list(m) == [0, 1, 0xFFFFFFFF]
    assert list(oracle.mutual_match(b, a, 0.0)) == [0, 1]
    assert list(oracle.mutual_match(a[:0], b, 0.8)) == []
    assert list(oracle.mutual_match(a, b[:0], 0.8)) == [0xFFFFFFFF] * 3
