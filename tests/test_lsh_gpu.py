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


def test_buckets_equal_reference_lsh_thread_sort_reduce(cuda_device):
    """The reference's own code + bucket grouping (FP16 hash GEMM, set_bit_h,
    thrust sort, host run-length) for the same hyperplanes."""
    import torch

    if not oracle.ref_available():
        pytest.skip("reference library not built")
    ref = oracle.ref()
    n, nbits = 4000, 16
    x = datagen.make_base(n, seed=77)
    rng = np.random.default_rng(3)
    planes = np.where(rng.random((nbits, 128)) >= 0.5, 1, -1).astype(np.int8)  # the reference's +/-1 family
    ours = ms.lsh_hash(torch.from_numpy(x).to(cuda_device), torch.from_numpy(planes[None]).to(cuda_device))
    ours = ours.cpu().numpy().view(np.uint32)[0]
    code = np.zeros(n, np.int32)
    index = np.zeros(n, np.int32)
    buckets = np.zeros(2 * n, np.int32)
    nb = ctypes.c_int(0)
    pts16 = x.astype(np.float16)
    pl16 = planes.astype(np.float16)
    rc = ref.ref_lsh_buckets(pts16.ctypes.data, n, pl16.ctypes.data, nbits, code.ctypes.data, index.ctypes.data,
                             buckets.ctypes.data, ctypes.byref(nb))
    assert rc == 0
    ref_code = code.view(np.uint32)
    dots = x.astype(np.int64) @ planes.astype(np.int64).T
    differ = ref_code != ours
    # The reference accumulates the hash GEMM in FP16: only points with a dot
    # product close to zero may land in another bucket.
    assert (np.abs(dots[differ]).min(axis=1) <= 64).all() if differ.any() else True
    assert differ.mean() < 0.01
    # identical grouping wherever the codes agree: the reference's sorted index
    # order groups equal codes contiguously
    assert (np.diff(ref_code[index].astype(np.int64)) >= 0).all()


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


@pytest.mark.parametrize("L,k,probes", [(2, 16, 1), (2, 16, 4), (1, 12, 16), (3, 10, 8)])
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
