"""Batched exact 2-NN (many uneven problems in one launch) through the C ABI.

Every problem's results must equal the oracle's for that problem alone, bit
for bit, whatever kernel shape runs, in one-shot calls and in CUDA-graph
replays of a plan.
"""
import numpy as np
import pytest

import matching_sift_b200 as ms
import oracle
from matching_sift_b200 import datagen

pytestmark = pytest.mark.gpu


def _uneven_batch(seed, n_pairs=24, hi=1500):
    """Query sets and base rows of problems with uneven sizes and edge cases
    (empty sets, one or two base rows, shared and overlapping base ranges)."""
    rng = np.random.default_rng([seed, 9])
    sizes = [(int(a), int(b)) for a, b in np.exp(rng.uniform(0, np.log(hi), (n_pairs, 2))).astype(int)]
    sizes += [(0, 50), (40, 0), (33, 1), (70, 2), (129, 129), (600, 257)]
    qs, bases, pairs = [], [], []
    r_rows = 0
    for k, (na, nb) in enumerate(sizes):
        b = datagen.make_base(nb, seed=seed * 1000 + k)
        a = (datagen.make_queries(na, b, seed=seed * 1000 + k, copy_frac=0.5 if nb else 0.0) if na
             else np.zeros((0, 128), np.uint8))
        qs.append(a)
        bases.append(b)
        pairs.append([na, nb, r_rows])
        r_rows += nb
    r = np.concatenate(bases) if bases else np.zeros((0, 128), np.uint8)
    # two problems reusing (parts of) earlier base rows
    if len(pairs) > 3 and r_rows > 10:
        for k, (off, nb) in enumerate([(pairs[1][2], pairs[1][1]), (3, min(400, r_rows - 3))]):
            a = datagen.make_queries(90 + k, r[off:off + nb] if nb else r[:1], seed=77 + k)
            qs.append(a)
            pairs.append([a.shape[0], nb, off])
    return np.concatenate(qs), r, np.array(pairs, np.uint32)


def _check_batch(q, r, pairs, out, threshold=0.8):
    idx = out["nn_idx"].cpu().numpy().astype(np.int64)
    dist = out["nn_dist"].cpu().numpy()
    m = out["matches"].cpu().numpy().view(np.uint32)
    a0 = 0
    for na, nb, off in pairs:
        na, nb, off = int(na), int(nb), int(off)
        sl = slice(a0, a0 + na)
        a0 += na
        if na == 0:
            continue
        d, i = oracle.brute_2nn_u8(q[sl], r[off:off + nb])
        np.testing.assert_array_equal(idx[sl], i, err_msg=f"pair {na}x{nb}@{off}")
        present = i >= 0
        np.testing.assert_array_equal(dist[sl][present].astype(np.int64), d[present])
        assert (dist[sl][~present] == np.finfo(np.float32).max).all()
        np.testing.assert_array_equal(m[sl], oracle.ratio_match(d, i, threshold))


def _dev(x, dev):
    import torch

    return torch.from_numpy(np.ascontiguousarray(x)).to(dev)


def test_one_shot_batch_vs_oracle(cuda_device):
    q, r, pairs = _uneven_batch(1)
    out = ms.match_batch(_dev(q, cuda_device), _dev(r, cuda_device), pairs)
    assert ms.stream_status() == ms.SIFT_OK
    _check_batch(q, r, pairs, out)


@pytest.mark.parametrize("shape", [0, 1, 2])
def test_plan_every_shape_vs_oracle(cuda_device, shape):
    q, r, pairs = _uneven_batch(2 + shape)
    plan = ms.BatchPlan(_dev(q, cuda_device), _dev(r, cuda_device), pairs, tune=False, shape=shape)
    info = plan.info()
    assert (info["qpt"], info["qbuf"]) == [(2, 1), (2, 2), (1, 2)][shape]
    out = plan.run()
    assert ms.stream_status() == ms.SIFT_OK
    _check_batch(q, r, pairs, out)
    plan.close()


def test_graph_replay_follows_new_data(cuda_device):
    import torch

    q, r, pairs = _uneven_batch(5)
    qd, rd = _dev(q, cuda_device), _dev(r, cuda_device)
    plan = ms.BatchPlan(qd, rd, pairs, tune=False)
    _check_batch(q, r, pairs, plan.run())
    # new descriptor values in the same buffers: the replayed graph reads them
    q2 = datagen.make_base(q.shape[0], seed=123)
    r2 = datagen.make_base(r.shape[0], seed=124)
    qd.copy_(torch.from_numpy(q2))
    rd.copy_(torch.from_numpy(r2))
    out = plan.run()
    torch.cuda.synchronize()
    _check_batch(q2, r2, pairs, out)
    for _ in range(3):
        out = plan.run()
    _check_batch(q2, r2, pairs, out)
    plan.close()


def test_autotuner_times_every_shape(cuda_device):
    q, r, pairs = _uneven_batch(6, n_pairs=40, hi=3000)
    plan = ms.BatchPlan(_dev(q, cuda_device), _dev(r, cuda_device), pairs, tune=True)
    info = plan.info()
    t = info["tuned_ms"]
    assert all(x > 0 for x in t), t
    shapes = [(2, 1), (2, 2), (1, 2)]
    assert t[shapes.index((info["qpt"], info["qbuf"]))] == min(t)
    _check_batch(q, r, pairs, plan.run())
    plan.close()
    # the one-shot call of a batch of the same sizes reuses the tuned shape
    out = ms.match_batch(_dev(q, cuda_device), _dev(r, cuda_device), pairs)
    _check_batch(q, r, pairs, out)


def test_empty_batches(cuda_device):
    import torch

    q = torch.zeros((0, 128), dtype=torch.uint8, device=cuda_device)
    r = torch.zeros((4, 128), dtype=torch.uint8, device=cuda_device)
    out = ms.match_batch(q, r, np.zeros((0, 3), np.uint32))
    assert out["nn_idx"].shape[0] == 0
    q = torch.zeros((5, 128), dtype=torch.uint8, device=cuda_device)
    out = ms.match_batch(q, r, [[5, 0, 0]])
    assert (out["nn_idx"].cpu().numpy() == -1).all()


def test_bad_pairs_are_rejected(cuda_device):
    import torch

    q = torch.zeros((5, 128), dtype=torch.uint8, device=cuda_device)
    r = torch.zeros((4, 128), dtype=torch.uint8, device=cuda_device)
    m = torch.zeros(5, dtype=torch.int32, device=cuda_device)
    pa = np.array([[5, 3, 2]], np.uint32)  # rows 2..4 of a 4-row base
    rc = ms.lib().sift2nn_match_batch(q.data_ptr(), r.data_ptr(), 4, pa.ctypes.data, 1, 0.8, m.data_ptr(), None,
                                      None, None)
    assert rc == ms.SIFT_ERR_INVALID_ARG


def test_image_pairs_workload_subset(cuda_device):
    """512 image pairs, 500..8000 keypoints per side (log-uniform), side B 40%
    noisy copies of side A: all distances recomputed from the returned indices,
    16 random pairs against the oracle."""
    pairs_data = datagen.make_pairs(512, seed=0)
    q = np.concatenate([a for a, _ in pairs_data])
    r = np.concatenate([b for _, b in pairs_data])
    pairs, off = [], 0
    for a, b in pairs_data:
        pairs.append([a.shape[0], b.shape[0], off])
        off += b.shape[0]
    pairs = np.array(pairs, np.uint32)
    plan = ms.BatchPlan(_dev(q, cuda_device), _dev(r, cuda_device), pairs, tune=True)
    out = plan.run()
    idx = out["nn_idx"].cpu().numpy().astype(np.int64)
    dist = out["nn_dist"].cpu().numpy().astype(np.int64)
    a0 = 0
    rng = np.random.default_rng(3)
    check = set(rng.choice(len(pairs), 16, replace=False).tolist())
    for k, (na, nb, boff) in enumerate(pairs.tolist()):
        sl = slice(a0, a0 + na)
        a0 += na
        base = r[boff:boff + nb].astype(np.int64)
        for c in range(2):
            dd = ((q[sl].astype(np.int64) - base[idx[sl, c]]) ** 2).sum(1)
            np.testing.assert_array_equal(dd, dist[sl, c])
        assert (dist[sl, 0] <= dist[sl, 1]).all()
        if k in check:
            d, i = oracle.brute_2nn_u8(q[sl], r[boff:boff + nb])
            np.testing.assert_array_equal(idx[sl], i)
    plan.close()
