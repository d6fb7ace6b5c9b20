"""LSH path on the GPU: codes, buckets and candidate scan against the oracle
and the reference's own bucketing (src/lsh_h.cu:565-629), through the C ABI."""
import ctypes

import numpy as np
import pytest

import matching_sift_b200 as ms
import oracle
from matching_sift_b200 import datagen

pytestmark = pytest.mark.gpu


def _planes(L, k, seed=0, scale=32.0):
    return datagen.quantize_planes(datagen.make_hyperplanes(k, L, seed=seed), scale)


@pytest.mark.parametrize("L,k", [(1, 12), (4, 16), (2, 24), (3, 7), (8, 24), (1, 32), (5, 1)])
def test_hash_codes_exact(cuda_device, L, k):
    import torch

    x = datagen.make_base(3000, seed=L * 100 + k)
    planes = _planes(L, k, seed=k)
    codes = ms.lsh_hash(torch.from_numpy(x).to(cuda_device), torch.from_numpy(planes).to(cuda_device))
    got = codes.cpu().numpy().view(np.uint32)
    for t in range(L):
        want, _ = oracle.lsh_codes(x, planes[t].astype(np.float32))
        np.testing.assert_array_equal(got[t], want, err_msg=f"table {t}")


@pytest.mark.parametrize("L,k", [(4, 12), (2, 20), (1, 8), (6, 16)])
def test_lsh_match_vs_oracle(cuda_device, L, k):
    import torch

    q, r = datagen.make_workload(1500, 30000, seed=k)
    planes = _planes(L, k, seed=L)
    out = ms.lsh_match(torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device),
                       torch.from_numpy(planes).to(cuda_device), threshold=0.8)
    assert ms.stream_status() == ms.SIFT_OK
    qc = np.stack([oracle.lsh_codes(q, planes[t].astype(np.float32))[0] for t in range(L)])
    rc = np.stack([oracle.lsh_codes(r, planes[t].astype(np.float32))[0] for t in range(L)])
    d, i = oracle.lsh_scan(q, r, qc, rc)
    np.testing.assert_array_equal(out["nn_idx"].cpu().numpy().astype(np.int64), i)
    present = i >= 0
    np.testing.assert_array_equal(out["nn_dist"].cpu().numpy()[present].astype(np.int64), d[present])
    want = oracle.ratio_match(np.where(present, d, np.iinfo(np.int64).max), i, 0.8)
    np.testing.assert_array_equal(out["matches"].cpu().numpy().view(np.uint32), want)


def _groups(codes, ids):
    """(code, id) pairs sorted lexicographically: the grouping as sets of ids per code."""
    o = np.lexsort((ids, codes))
    return np.stack([codes[o].astype(np.int64), ids[o].astype(np.int64)])


# Unit roundoff of FP16 and the worst-case bound of a 128-term FP16 sum
# (products and partial sums each rounded): |fl(sum) - sum| <= gamma_128 * sum |x_i p_i|.
_U16 = 2.0 ** -11
_GAMMA128 = 128 * _U16 / (1 - 128 * _U16)


@pytest.mark.parametrize("family", ["pm1", "gauss"])
@pytest.mark.parametrize("k", [12, 16, 20, 24])
def test_buckets_equal_reference_lsh_thread_sort_reduce(cuda_device, family, k):
    """Bucket contents against the reference's own bucketing given the same
    hyperplanes (lsh_thread_sort_reduce, src/lsh_h.cu:565-629: cublasHgemm hash
    dots as at :909, set_bit_h, thrust sort by code, host run-length into
    {first id, count} runs), 100,000 generator points.

    Hyperplane families: the reference's own +/-1 planes (pm1), and N(0,1)
    planes rounded to multiples of 1/32 (gauss: exact in FP16 for the
    reference, int8 x 1/32 here), so both sides hash with identical planes.
    The library's dot products are exact integers; the reference's are FP16
    sums. Every point whose code differs is listed, and each of its differing
    bits must have |exact dot| within the FP16 bound gamma_128 * sum|x_i p_i|.
    Apart from those points the two groupings are identical as sets of ids per
    code, and the reference's runs are checked to be its groups."""
    import torch

    if not oracle.ref_available():
        pytest.skip("reference library not built")
    ref = oracle.ref()
    n = 100_000
    x = datagen.make_base(n, seed=77)
    rng = np.random.default_rng(1000 + k)
    if family == "pm1":
        planes = np.where(rng.random((k, 128)) >= 0.5, 1, -1).astype(np.int8)
        pl16 = planes.astype(np.float16)
    else:
        planes = datagen.quantize_planes(datagen.make_hyperplanes(k, 1, seed=k), 32.0)[0]
        pl16 = (planes.astype(np.float32) / 32.0).astype(np.float16)
        assert np.array_equal(pl16.astype(np.float32) * 32.0, planes.astype(np.float32))
    xd = torch.from_numpy(x).to(cuda_device)
    codes = ms.lsh_hash(xd, torch.from_numpy(planes[None]).to(cuda_device))
    start, order, ocode = ms.lsh_buckets(codes, k)
    ours = codes.cpu().numpy().view(np.uint32)[0]
    start, order, ocode = start.cpu().numpy()[0], order.cpu().numpy()[0], ocode.cpu().numpy().view(np.uint32)[0]

    code = np.zeros(n, np.int32)
    index = np.zeros(n, np.int32)
    buckets = np.zeros(2 * n, np.int32)
    nb = ctypes.c_int(0)
    x16 = np.ascontiguousarray(x.astype(np.float16))  # held for the call: a temporary would be freed first
    rc = ref.ref_lsh_buckets(x16.ctypes.data, n, pl16.ctypes.data, k, code.ctypes.data,
                             index.ctypes.data, buckets.ctypes.data, ctypes.byref(nb))
    assert rc == 0
    ref_code = code.view(np.uint32)
    runs = buckets[:2 * nb.value].reshape(-1, 2)

    # The library: exact codes, and its table groups every point by its code.
    dots = x.astype(np.int64) @ planes.astype(np.int64).T
    exact = ((dots < 0).astype(np.uint64) << np.arange(k, dtype=np.uint64)).sum(1).astype(np.uint32)
    np.testing.assert_array_equal(ours, exact)
    top = min(k, 16)
    assert start[0] == 0 and start[-1] == n and (np.diff(start) >= 0).all()
    np.testing.assert_array_equal(ocode, ours[order])
    np.testing.assert_array_equal(np.repeat(np.arange(1 << top), np.diff(start)), ocode >> (k - top))

    # The reference: its runs partition its sorted index into groups of one code.
    assert runs[:, 1].sum() == n and (runs[:, 1] > 0).all()
    pos = np.concatenate([[0], np.cumsum(runs[:, 1])[:-1]])
    np.testing.assert_array_equal(index[pos], runs[:, 0])  # each run starts at its first id
    run_code = ref_code[runs[:, 0]]
    np.testing.assert_array_equal(ref_code[index], np.repeat(run_code, runs[:, 1]))
    assert len(np.unique(run_code)) == len(run_code)
    assert sorted(index.tolist()) == list(range(n))

    # Differences: points whose FP16 code differs, every differing bit within the bound.
    differ = np.nonzero(ref_code != ours)[0]
    bound = _GAMMA128 * (x.astype(np.float64) @ np.abs(planes.astype(np.float64)).T)
    for i in differ:
        bits = np.nonzero((int(ref_code[i]) ^ int(ours[i])) >> np.arange(k) & 1)[0]
        assert (np.abs(dots[i, bits]) <= bound[i, bits]).all(), (i, bits, dots[i, bits], bound[i, bits])
    near = (np.abs(dots) <= bound).any(1)
    assert len(differ) <= int(near.sum())
    # How tight the explanation is: the largest |dot| / sum|x_i p_i| of a
    # differing bit, and how many points have some bit at least that close to 0.
    rel = np.abs(dots) / np.maximum(x.astype(np.float64) @ np.abs(planes.astype(np.float64)).T, 1.0)
    worst = max((rel[i][(int(ref_code[i]) ^ int(ours[i])) >> np.arange(k) & 1 == 1].max() for i in differ),
                default=0.0)
    close = int((rel <= worst).any(1).sum()) if len(differ) else 0
    print(f"{family} k={k}: {len(differ)} of {n} points hashed differently by the FP16 reference "
          f"(points with a bit inside the FP16 bound: {int(near.sum())}); largest |dot| / sum|x p| of a differing "
          f"bit {worst:.2e}, points with a bit that close to 0: {close}; buckets {nb.value}")

    # Identical groupings apart from those points.
    keep = np.ones(n, bool)
    keep[differ] = False
    ids = np.arange(n)
    np.testing.assert_array_equal(_groups(ref_code[keep], ids[keep]), _groups(ours[keep], ids[keep]))
    # ... and each differing point sits in the group of its own code on each side.
    in_ours = np.zeros(n, np.uint32)
    in_ours[order] = ocode
    in_ref = np.zeros(n, np.uint32)
    in_ref[index] = np.repeat(run_code, runs[:, 1])
    np.testing.assert_array_equal(in_ours[differ], ours[differ])
    np.testing.assert_array_equal(in_ref[differ], ref_code[differ])


def test_lsh_gpu_reference_entry_point(cuda_device):
    """lsh_gpu draws +/-1 hyperplanes with libc rand() in the reference's order."""
    import torch

    libc = ctypes.CDLL("libc.so.6")
    q, r = datagen.make_workload(800, 20000, seed=8)
    L, nbits = 3, 10
    libc.srand(1234)
    planes = np.empty((L, nbits, 128), np.int8)
    rand_max = np.float32(2147483647)
    for t in range(L):
        for j in range(nbits):
            for d in range(128):
                v = np.float32(libc.rand()) / rand_max
                planes[t, j, d] = 1 if float(v) - 0.5 >= 0 else -1
    qf = torch.from_numpy(q.astype(np.float32)).to(cuda_device)
    rf = torch.from_numpy(r.astype(np.float32)).to(cuda_device)
    m = torch.zeros(800, dtype=torch.int32, device=cuda_device)
    libc.srand(1234)
    assert ms.lsh_gpu(qf, rf, ms.FLOAT_DEVICE, 800, 20000, m, 0.8, None, 2, L, 0, nbits) == ms.SIFT_OK
    want = ms.lsh_match(torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device),
                        torch.from_numpy(planes).to(cuda_device), threshold=0.0)
    np.testing.assert_array_equal(m.cpu().numpy(), want["matches"].cpu().numpy())


def test_lsh_recall_against_exact(cuda_device):
    import torch

    q, r = datagen.make_workload(2000, 100000, seed=9)
    qt, rt = torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)
    exact = ms.match(qt, rt, outputs=("nn_idx",))["nn_idx"].cpu().numpy()[:, 0]
    lsh = ms.lsh_match(qt, rt, torch.from_numpy(_planes(8, 12)).to(cuda_device))["nn_idx"].cpu().numpy()[:, 0]
    recall = (lsh == exact).mean()
    assert recall > 0.5, recall


def _probe_codes(codes, dots, k, probes):
    """Query-directed probes of one table: the min(6, k) lowest-margin bits
    (|q . plane|, ties by bit index), their subsets by summed margin (ties by
    subset id), the first `probes` applied to the code."""
    flip = min(6, k)
    out = np.empty((probes, len(codes)), np.uint32)
    for i in range(len(codes)):
        mag = np.abs(dots[i, :k])
        kept = sorted(range(k), key=lambda j: (mag[j], j))[:flip]
        subsets = sorted(range(1 << flip), key=lambda s: (sum(mag[kept[b]] for b in range(flip) if s >> b & 1), s))
        for p in range(probes):
            c = int(codes[i])
            for b in range(flip):
                if subsets[p] >> b & 1:
                    c ^= 1 << kept[b]
            out[p, i] = c
    return out


# (1, 14, 40) and (2, 12, 64): more probes per table than a warp has lanes
# (the scan fetches a table's probes one per lane, two per lane past 32).
@pytest.mark.parametrize("L,k,probes", [(2, 16, 1), (2, 16, 4), (1, 12, 16), (3, 10, 8), (1, 14, 40), (2, 12, 64)])
def test_multiprobe_vs_oracle(cuda_device, L, k, probes):
    import torch

    q, r = datagen.make_workload(1200, 30000, seed=probes + k)
    planes = _planes(L, k, seed=L + probes)
    out = ms.lsh_match(torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device),
                       torch.from_numpy(planes).to(cuda_device), threshold=0.8, probes=probes, candidates=True)
    assert ms.stream_status() == ms.SIFT_OK
    qcodes, rcodes, cand = [], [], np.zeros(q.shape[0], np.int64)
    for t in range(L):
        qc, qdots = oracle.lsh_codes(q, planes[t].astype(np.float32))
        rc, _ = oracle.lsh_codes(r, planes[t].astype(np.float32))
        pc = _probe_codes(qc, qdots, k, probes)
        sizes = dict(zip(*np.unique(rc, return_counts=True)))
        for i in range(q.shape[0]):
            cand[i] += sum(int(sizes.get(c, 0)) for c in set(pc[:, i].tolist()))
        qcodes.append(pc)
        rcodes.extend([rc] * probes)
    d, i = oracle.lsh_scan(q, r, np.concatenate(qcodes), np.stack(rcodes))
    np.testing.assert_array_equal(out["nn_idx"].cpu().numpy().astype(np.int64), i)
    present = i >= 0
    np.testing.assert_array_equal(out["nn_dist"].cpu().numpy()[present].astype(np.int64), d[present])
    want = oracle.ratio_match(np.where(present, d, np.iinfo(np.int64).max), i, 0.8)
    np.testing.assert_array_equal(out["matches"].cpu().numpy().view(np.uint32), want)
    np.testing.assert_array_equal(out["candidates"].cpu().numpy().astype(np.int64), cand)


def test_more_probes_never_lose_the_nearest(cuda_device):
    import torch

    q, r = datagen.make_workload(2000, 100000, seed=3)
    planes = torch.from_numpy(_planes(4, 16, seed=9)).to(cuda_device)
    qd, rd = torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)
    exact = ms.match(qd, rd, outputs=("nn_idx",))["nn_idx"][:, 0].cpu().numpy()
    prev_d, prev_hits = None, -1
    for probes in (1, 2, 8, 32):
        o = ms.lsh_match(qd, rd, planes, probes=probes, candidates=True)
        d1 = o["nn_dist"][:, 0].cpu().numpy()
        hits = int((o["nn_idx"][:, 0].cpu().numpy() == exact).sum())
        if prev_d is not None:
            assert (d1 <= prev_d).all()
            assert hits >= prev_hits
        prev_d, prev_hits = d1, hits
    assert prev_hits > 0
    with pytest.raises(ms.SiftError):
        ms.lsh_match(qd, rd, planes, probes=65)
