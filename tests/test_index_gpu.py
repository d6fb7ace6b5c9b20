"""Persistent hash indexes (sift_lsh_index_create / sift_mlp_index_create /
sift_index_search), through the C ABI: one bucketing of the base, many
searches, each equal to the oracle's scan of the same buckets and to the
per-call entry points (sift_lsh_match_probes, sift_mlp_match)."""
import numpy as np
import pytest

import matching_sift_b200 as ms
import oracle
from matching_sift_b200 import datagen
from oracle import learned_hash as lh

pytestmark = pytest.mark.gpu


def _dev(x, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x)).to(dev)


def _same(a, b, keys=("matches", "nn_idx", "nn_dist", "candidates")):
    for k in keys:
        np.testing.assert_array_equal(a[k].cpu().numpy(), b[k].cpu().numpy(), err_msg=k)


@pytest.mark.parametrize("L,k,probes", [(1, 12, 1), (4, 16, 1), (2, 20, 4), (3, 24, 8)])
def test_lsh_index_equals_oracle_and_per_call(cuda_device, L, k, probes):
    q, r = datagen.make_workload(1500, 40000, seed=k + L)
    planes = datagen.quantize_planes(datagen.make_hyperplanes(k, L, seed=k), 32.0)
    qd, rd, pd = _dev(q, cuda_device), _dev(r, cuda_device), _dev(planes, cuda_device)
    idx = ms.HashIndex.lsh(rd, pd)
    per_call = ms.lsh_match(qd, rd, pd, threshold=0.8, probes=probes, candidates=True)
    for _ in range(2):  # searched twice: the index is reused as built
        got = idx.search(qd, probes=probes, threshold=0.8)
        assert ms.stream_status() == ms.SIFT_OK
        _same(got, per_call)
    if probes == 1:
        qc = np.stack([oracle.lsh_codes(q, planes[t].astype(np.float32))[0] for t in range(L)])
        rc = np.stack([oracle.lsh_codes(r, planes[t].astype(np.float32))[0] for t in range(L)])
        d, i = oracle.lsh_scan(q, r, qc, rc)
        np.testing.assert_array_equal(got["nn_idx"].cpu().numpy().astype(np.int64), i)
        present = i >= 0
        np.testing.assert_array_equal(got["nn_dist"].cpu().numpy()[present].astype(np.int64), d[present])
    idx.close()


def test_lsh_index_buckets_are_the_codes_groups(cuda_device):
    """The index's bucket table groups exactly the base's codes (as sets)."""
    import torch

    L, k = 2, 20
    r = datagen.make_base(30000, seed=3)
    planes = datagen.quantize_planes(datagen.make_hyperplanes(k, L, seed=4), 32.0)
    idx = ms.HashIndex.lsh(_dev(r, cuda_device), _dev(planes, cuda_device))
    start, order, ocode, top = idx.buckets()
    torch.cuda.synchronize()
    assert top == 16
    n, nb = r.shape[0], (1 << top) + 1
    s, o, c = start.cpu().numpy(), order.cpu().numpy(), ocode.cpu().numpy().view(np.uint32)
    for t in range(L):
        codes, _ = oracle.lsh_codes(r, planes[t].astype(np.float32))
        assert s[t, 0] == 0 and s[t, -1] == n
        assert sorted(o[t].tolist()) == list(range(n))
        np.testing.assert_array_equal(c[t], codes[o[t]])
        grp = np.repeat(np.arange(nb - 1), np.diff(s[t]))
        np.testing.assert_array_equal(grp, c[t] >> (k - top))


def test_mlp_index_equals_per_call_match(cuda_device):
    k = 16
    p = lh.init_params(k, seed=21)
    model = ms.MlpHash.from_params(_dev(p, cuda_device), k)
    q, r = datagen.make_workload(2000, 50000, seed=22)
    qd, rd = _dev(q, cuda_device), _dev(r, cuda_device)
    idx = ms.HashIndex.mlp(rd, model)
    for probes, min_cand, max_dist in ((1, 0, 0.0), (8, 0, 0.0), (4, 64, 0.0), (2, 0, 20000.0)):
        want = model.match(qd, rd, n_probes=probes, min_candidates=min_cand, max_dist=max_dist, threshold=0.8)
        got = idx.search(qd, probes=probes, min_candidates=min_cand, max_dist=max_dist, threshold=0.8)
        assert ms.stream_status() == ms.SIFT_OK
        _same(got, want)
        assert got["fallback"] == want["fallback"]
    # every query sent to the exact fallback: equal to the exact oracle
    got = idx.search(qd, probes=1, min_candidates=10 ** 9, threshold=0.8)
    assert got["fallback"] == q.shape[0]
    d, i = oracle.brute_2nn_u8(q, r)
    np.testing.assert_array_equal(got["nn_idx"].cpu().numpy().astype(np.int64), i)
    np.testing.assert_array_equal(got["nn_dist"].cpu().numpy().astype(np.int64), d)
    idx.close()


def test_index_arguments_are_checked(cuda_device):
    planes = _dev(datagen.quantize_planes(datagen.make_hyperplanes(12, 1, seed=1), 32.0), cuda_device)
    r = _dev(datagen.make_base(1000, seed=1), cuda_device)
    idx = ms.HashIndex.lsh(r, planes)
    with pytest.raises(ms.SiftError):
        idx.search(r[:10], probes=65)
    with pytest.raises(ms.SiftError):
        idx.search(r[:10], probes=0)
    out = idx.search(r[:0])
    assert out["fallback"] == 0
    idx.close()
    with pytest.raises(ms.SiftError):
        ms.HashIndex.lsh(r, _dev(np.zeros((9, 32, 128), np.int8), cuda_device))  # L * k > 256
