"""Learned hash on the GPU against its FP64 oracle (oracle/learned_hash.py).

* one training step's loss and gradients (hand-written forward / backward
  kernels) against the FP64 restatement;
* the tensor-core inference kernel's z and codes against the restatement;
* matching: with every bucket probed, or every query sent to the exact
  fallback, the results equal the exact oracle's bit for bit;
* training: deterministic for a seed, lowers the loss, and makes a query
  share its code with its true nearest neighbour far more often than with a
  random base row.
"""
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


def _rows(B, seed):
    base = datagen.make_base(4 * B, seed=seed)
    q = datagen.make_queries(B, base, seed=seed)
    return np.concatenate([q, base[:B], base[2 * B:3 * B]])


@pytest.mark.parametrize("k", [8, 16, 32])
def test_loss_and_gradients_match_fp64(cuda_device, k):
    B = 96
    x = _rows(B, k)
    p = lh.init_params(k, seed=k)
    loss, g = ms.mlp_loss_grad(_dev(x, cuda_device), B, k, _dev(p, cuda_device), 0.8, 0.6)
    want_loss, want_g = lh.loss_grad(p, x, B, k, 0.8, 0.6)
    np.testing.assert_allclose(loss, want_loss, rtol=2e-4, atol=1e-6)
    g = g.cpu().numpy().astype(np.float64)
    o = [0, lh.HID * lh.IN, lh.HID * lh.IN + lh.HID, lh.HID * lh.IN + lh.HID + lh.OUT_ROWS * lh.HID, lh.N_PARAMS]
    for name, a, b in zip(("W1", "b1", "W2", "b2"), o[:-1], o[1:]):
        err = np.linalg.norm(g[a:b] - want_g[a:b]) / max(np.linalg.norm(want_g[a:b]), 1e-12)
        assert err < 2e-3, (name, err)  # FP32 GPU arithmetic vs FP64


@pytest.mark.parametrize("k", [12, 32])
def test_inference_codes_match_fp64(cuda_device, k):
    import torch

    p = lh.init_params(k, seed=100 + k)
    model = ms.MlpHash.from_params(_dev(p, cuda_device), k)
    x = datagen.make_base(5000, seed=7)
    codes, z = model.hash(_dev(x, cuda_device), with_z=True)
    torch.cuda.synchronize()
    assert ms.stream_status() == ms.SIFT_OK
    _, zr = lh.forward(p, x, k)
    z = z.cpu().numpy().astype(np.float64)
    assert np.abs(z - zr).max() < 5e-3 * max(1.0, np.abs(zr).max())
    got = codes.cpu().numpy().view(np.uint32)
    bits_got = (got[:, None] >> np.arange(k)) & 1
    bits_ref = (zr > 0).astype(np.uint32)
    clear = np.abs(zr) > 1e-2
    np.testing.assert_array_equal(bits_got[clear], bits_ref[clear])
    # code bits follow the kernel's own z exactly
    np.testing.assert_array_equal(bits_got, (z > 0).astype(np.uint32))


def test_every_bucket_probed_equals_exact(cuda_device):
    """k = 4 bits and 16 probes: every code is probed, every base row is a
    candidate, so the result is the exact 2-NN (and ratio test)."""
    k = 4
    model = ms.MlpHash.from_params(_dev(lh.init_params(k, seed=3), cuda_device), k)
    q, r = datagen.make_workload(700, 6000, seed=21)
    out = model.match(_dev(q, cuda_device), _dev(r, cuda_device), n_probes=16, threshold=0.8)
    d, i = oracle.brute_2nn_u8(q, r)
    np.testing.assert_array_equal(out["nn_idx"].cpu().numpy().astype(np.int64), i)
    np.testing.assert_array_equal(out["nn_dist"].cpu().numpy().astype(np.int64), d)
    np.testing.assert_array_equal(out["matches"].cpu().numpy().view(np.uint32), oracle.ratio_match(d, i, 0.8))
    assert (out["candidates"].cpu().numpy() == r.shape[0]).all()
    assert out["fallback"] == 0


def test_fallback_to_exact(cuda_device):
    k = 20
    model = ms.MlpHash.from_params(_dev(lh.init_params(k, seed=4), cuda_device), k)
    q, r = datagen.make_workload(900, 5000, seed=22)
    out = model.match(_dev(q, cuda_device), _dev(r, cuda_device), n_probes=1, min_candidates=1 << 30, threshold=0.8)
    assert out["fallback"] == 900
    d, i = oracle.brute_2nn_u8(q, r)
    np.testing.assert_array_equal(out["nn_idx"].cpu().numpy().astype(np.int64), i)
    np.testing.assert_array_equal(out["nn_dist"].cpu().numpy().astype(np.int64), d)
    np.testing.assert_array_equal(out["matches"].cpu().numpy().view(np.uint32), oracle.ratio_match(d, i, 0.8))
    # partial fallback (8 bits: buckets of a few dozen rows): the queries below
    # the candidate floor get the exact answer, every other answer is a real
    # candidate at its exact distance, never better than the true nearest
    model = ms.MlpHash.from_params(_dev(lh.init_params(8, seed=4), cuda_device), 8)
    out = model.match(_dev(q, cuda_device), _dev(r, cuda_device), n_probes=4, min_candidates=64)
    cand = out["candidates"].cpu().numpy()
    low = cand < 64
    assert out["fallback"] == low.sum() and 0 < low.sum() < 900
    idx = out["nn_idx"].cpu().numpy().astype(np.int64)
    dist = out["nn_dist"].cpu().numpy().astype(np.int64)
    np.testing.assert_array_equal(idx[low], i[low])
    np.testing.assert_array_equal(dist[low], d[low])
    has = idx[:, 0] >= 0
    dd = ((q[has].astype(np.int64) - r[idx[has, 0]].astype(np.int64)) ** 2).sum(1)
    np.testing.assert_array_equal(dd, dist[has, 0])
    assert (dist[has, 0] >= d[has, 0]).all()
    # distance criterion: a query whose nearest candidate is farther than
    # max_dist (or that found none) gets the exact answer; the rest keep theirs
    plain = model.match(_dev(q, cuda_device), _dev(r, cuda_device), n_probes=4)["nn_dist"].cpu().numpy()
    out2 = model.match(_dev(q, cuda_device), _dev(r, cuda_device), n_probes=4, max_dist=40000.0)
    far = ~(plain[:, 0].astype(np.float64) <= 40000.0)
    assert out2["fallback"] == far.sum() and 0 < far.sum() < 900
    idx2 = out2["nn_idx"].cpu().numpy().astype(np.int64)
    np.testing.assert_array_equal(idx2[far], i[far])
    np.testing.assert_array_equal(out2["nn_dist"].cpu().numpy()[far].astype(np.int64), d[far])


def test_training_is_deterministic_and_learns(cuda_device):
    import torch

    base = datagen.make_base(60000, seed=31)
    tq = datagen.make_queries(8000, base, seed=32)
    held = datagen.make_queries(1500, base, seed=33)
    bd, td, hd = _dev(base, cuda_device), _dev(tq, cuda_device), _dev(held, cuda_device)
    k = 12
    m1 = ms.MlpHash.train(bd, td, k=k, steps=150, batch=512, lr=3e-3, seed=5)
    m2 = ms.MlpHash.train(bd, td, k=k, steps=150, batch=512, lr=3e-3, seed=5)
    assert torch.equal(m1.params, m2.params)
    c = m1.loss_curve
    assert np.isfinite(c).all() and c[-20:].mean() < c[:5].mean()
    # Selectivity: how much more often a held-out query shares its code with
    # its true nearest neighbour than with a random base row.
    _, i_true = oracle.brute_2nn_u8(held, base)
    rnd = np.random.default_rng(9).integers(0, base.shape[0], 200)
    untrained = ms.MlpHash.from_params(_dev(lh.init_params(k, seed=5), cuda_device), k)
    sel = {}
    for name, m in (("trained", m1), ("untrained", untrained)):
        cq = m.hash(hd).cpu().numpy()
        cb = m.hash(bd).cpu().numpy()
        same_nn = (cq == cb[i_true[:, 0]]).mean()
        same_rand = (cq[:, None] == cb[None, rnd]).mean()
        sel[name] = same_nn / max(same_rand, 1e-6)
    assert sel["trained"] > 2 * sel["untrained"], sel


def test_trained_hash_beats_random_hyperplanes_at_equal_work(cuda_device):
    """What the network gains over the method it replaces: held-out recall@1
    of the learned hash against random-hyperplane LSH (the reference's family,
    src/lsh_h.cu:51-100; N(0,1) planes here, one table), both with 16 bits and
    through a persistent index of the same base, at equal work: for every LSH
    operating point (probes 1, 4, 16), the learned hash with the most probes
    whose mean candidate count does not exceed LSH's must find the true
    nearest neighbour more often. (At equal probes the trained hash is far
    more selective -- its buckets are balanced by the loss -- so it compares
    many fewer candidates.) The gain is asserted on the noisy-copy half of the
    queries, whose nearest neighbour is well separated (the fresh half have
    no close neighbour for any hash to find), by at least 0.05 at LSH's 1 and
    4 probes, where its recall over all queries must be higher too; at 16
    probes both find nearly every copy and the learned hash must not be worse
    on them. (Over all queries at 16 probes LSH compares 4x more candidates
    than the learned hash at its 64-probe maximum and picks up a few more
    fresh draws by chance, so the overall recall is not compared there.)"""
    base = datagen.make_base(100_000, seed=41)
    tq = datagen.make_queries(20_000, base, seed=42)
    held = datagen.make_queries(3000, base, seed=43)
    copies = datagen.query_copies(3000, seed=43)
    bd, td, hd = _dev(base, cuda_device), _dev(tq, cuda_device), _dev(held, cuda_device)
    _, i_true = oracle.brute_2nn_u8(held, base)
    k = 16
    model = ms.MlpHash.train(bd, td, k=k, steps=600, batch=1024, lr=2e-3, seed=3)
    learned = ms.HashIndex.mlp(bd, model)
    planes = datagen.quantize_planes(datagen.make_hyperplanes(k, 1, seed=44), 32.0)
    lsh = ms.HashIndex.lsh(bd, _dev(planes, cuda_device))

    def point(idx, probes):
        out = idx.search(hd, probes=probes)
        hit = out["nn_idx"][:, 0].cpu().numpy() == i_true[:, 0]
        return {"probes": probes, "recall": float(hit.mean()), "recall_copies": float(hit[copies].mean()),
                "candidates": float(out["candidates"].double().mean().item())}

    curve = [point(learned, p) for p in (1, 2, 4, 8, 16, 32, 64)]
    for probes in (1, 4, 16):
        ref = point(lsh, probes)
        cheaper = [c for c in curve if c["candidates"] <= ref["candidates"]]
        assert cheaper, (ref, curve)
        best = cheaper[-1]
        print("lsh", ref, "learned", best)
        # at 16 probes both find nearly every noisy copy: not worse there
        margin = 0.05 if probes < 16 else 0.0
        assert best["recall_copies"] >= ref["recall_copies"] + margin, (ref, best)
        if probes < 16:
            assert best["recall"] >= ref["recall"], (ref, best)
    learned.close()
    lsh.close()
