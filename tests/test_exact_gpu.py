"""Parity of the CUDA exact path with the oracle and the reference, through the C ABI.

Exact path results are integers, so every comparison is bit-exact: nearest and
second-nearest indices (lexicographic ties, lower index first) and squared
distances.
"""
import glob
import os

import numpy as np
import pytest

import matching_sift_b200 as ms
import oracle
from matching_sift_b200 import datagen

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FLT_MAX = np.float32(np.finfo(np.float32).max)


KERNELS = {"fold": 0, "single": 1, "pair": 3}


@pytest.fixture(params=sorted(KERNELS))
def kernel(request):
    """Runs a test once per exact-search kernel (CTA-pair with folded norms, single-CTA, CTA-pair)."""
    ms.lib().sift_set_kernel_variant(KERNELS[request.param])
    yield request.param
    ms.lib().sift_set_kernel_variant(0)


def _run(q, r, dev, metric=ms.METRIC_L2, threshold=0.8):
    import torch

    qt = torch.from_numpy(np.ascontiguousarray(q)).to(dev)
    rt = torch.from_numpy(np.ascontiguousarray(r)).to(dev)
    out = ms.match(qt, rt, threshold=threshold, metric=metric, outputs=("matches", "nn_idx", "nn_dist", "sorted"))
    assert ms.stream_status() == ms.SIFT_OK
    return {k: v.cpu().numpy() for k, v in out.items()}


def _check_against_oracle(q, r, got, metric=ms.METRIC_L2):
    d, i = oracle.brute_2nn_u8(q, r, metric=metric)
    np.testing.assert_array_equal(got["nn_idx"].astype(np.int64), i)
    present = i >= 0
    qn = (q.astype(np.int64) ** 2).sum(1) if metric == ms.METRIC_L2 else None
    np.testing.assert_array_equal(got["nn_dist"][present].astype(np.int64), d[present])
    assert (got["nn_dist"][~present] == FLT_MAX).all()
    return d, i, qn


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "host_brute_*.npz"))), ids=os.path.basename)
def test_golden_host_brute(cuda_device, kernel, path):
    z = np.load(path)
    q, r, ref = z["q"], z["r"], z["sorted"]
    got = _run(q, r, cuda_device)
    np.testing.assert_array_equal(got["sorted"], ref)


@pytest.mark.parametrize("metric", [ms.METRIC_L2, ms.METRIC_DOT])
def test_config1_vs_oracle(cuda_device, kernel, metric):
    """1,000 queries x 10,000 base rows from the seeded generator."""
    q, r = datagen.make_workload(1000, 10000, seed=0)
    got = _run(q, r, cuda_device, metric=metric)
    d, i, _ = _check_against_oracle(q, r, got, metric)
    if metric == ms.METRIC_L2:
        np.testing.assert_array_equal(got["matches"], oracle.ratio_match(d, i, 0.8))


@pytest.mark.parametrize("q_n,r_n", [(1, 1), (1, 2), (3, 300), (127, 255), (128, 256), (129, 257), (255, 513),
                                     (256, 1000), (300, 4097), (1000, 77), (2048, 1)])
def test_ragged_sizes(cuda_device, kernel, q_n, r_n):
    q, r = datagen.make_workload(q_n, r_n, seed=q_n * 7 + r_n)
    got = _run(q, r, cuda_device)
    _check_against_oracle(q, r, got)


def test_ties_choose_lower_index(cuda_device, kernel):
    base = datagen.make_base(300, seed=1)
    r = np.concatenate([base, base, base], axis=0)  # every row three times
    q = np.concatenate([base[::3], datagen.make_base(50, seed=2)], axis=0)
    got = _run(q, r, cuda_device)
    d, i, _ = _check_against_oracle(q, r, got)
    assert (got["nn_idx"][:100, 0] == np.arange(0, 300, 3)).all()
    assert (got["nn_idx"][:100, 1] == np.arange(0, 300, 3) + 300).all()


def test_extreme_values(cuda_device, kernel):
    r = np.stack([np.zeros(128, np.uint8), np.full(128, 255, np.uint8)] * 200)
    q = np.stack([np.full(128, 255, np.uint8), np.zeros(128, np.uint8), np.full(128, 128, np.uint8)] * 50)
    got = _run(q, r, cuda_device)
    _check_against_oracle(q, r, got)
    assert got["nn_dist"][0, 0] == 0 and got["nn_dist"][2, 0] == 128 * 127 ** 2


def test_device_types_refuse_host_pointers(cuda_device):
    """A host array passed as device memory is refused (SIFT_ERR_INVALID_ARG)
    before it can reach a tensor map or a kernel."""
    import torch

    q, r = datagen.make_workload(64, 256, seed=5)
    qd = torch.from_numpy(q).to(cuda_device)
    rd = torch.from_numpy(r).to(cuda_device)
    m = torch.empty(64, dtype=torch.int32, device=cuda_device)
    st = torch.cuda.current_stream(cuda_device).cuda_stream
    lib = ms.lib()
    qh = np.ascontiguousarray(q)
    rh = np.ascontiguousarray(r)
    for qp, rp in ((qh.ctypes.data, rd.data_ptr()), (qd.data_ptr(), rh.ctypes.data)):
        rc = lib.sift2nn_match(qp, rp, ms.U8_DEVICE, 64, 256, ms.METRIC_L2, 0.8, m.data_ptr(), None, None, None, st)
        assert rc == ms.SIFT_ERR_INVALID_ARG
    qf = np.ascontiguousarray(q.astype(np.float32))
    rf = rd.float()
    rc = lib.sift2nn_match(qf.ctypes.data, rf.data_ptr(), ms.FLOAT_DEVICE, 64, 256, ms.METRIC_L2, 0.8,
                           m.data_ptr(), None, None, None, st)
    assert rc == ms.SIFT_ERR_INVALID_ARG
    assert ms.stream_status() == ms.SIFT_OK


def test_no_base_rows(cuda_device):
    import torch

    q = torch.zeros((5, 128), dtype=torch.uint8, device=cuda_device)
    r = torch.zeros((0, 128), dtype=torch.uint8, device=cuda_device)
    out = ms.match(q, r, outputs=("matches", "nn_idx", "nn_dist"))
    assert (out["nn_idx"].cpu().numpy() == -1).all()
    assert (out["matches"].cpu().numpy().astype(np.int64) & 0xFFFFFFFF == 0xFFFFFFFF).all()


def test_scale_subset_vs_oracle(cuda_device, kernel):
    """10,000 x 1,000,000: 96 random queries checked against the oracle, all
    queries checked by recomputing both distances from the returned indices."""
    q, r = datagen.make_workload(10000, 1000000, seed=0)
    got = _run(q, r, cuda_device)
    rng = np.random.default_rng(1)
    sel = np.sort(rng.choice(q.shape[0], 96, replace=False))
    d, i = oracle.brute_2nn_u8(q[sel], r)
    np.testing.assert_array_equal(got["nn_idx"][sel].astype(np.int64), i)
    np.testing.assert_array_equal(got["nn_dist"][sel].astype(np.int64), d)
    idx = got["nn_idx"].astype(np.int64)
    assert (idx >= 0).all() and (idx < r.shape[0]).all() and (idx[:, 0] != idx[:, 1]).all()
    for k in range(2):
        dd = ((q.astype(np.int64) - r[idx[:, k]].astype(np.int64)) ** 2).sum(1)
        np.testing.assert_array_equal(dd, got["nn_dist"][:, k].astype(np.int64))
    assert (got["nn_dist"][:, 0] <= got["nn_dist"][:, 1]).all()


# ------------------------------------------------- reference-named entry points

def test_cublas_2nn_sift_all_memory_types(cuda_device):
    import torch

    q, r = datagen.make_workload(500, 3000, seed=5)
    d, i = oracle.brute_2nn_u8(q, r)
    want = oracle.ratio_match(d, i, 0.8)
    qf, rf = q.astype(np.float32), r.astype(np.float32)
    inputs = {
        ms.FLOAT_DEVICE: (torch.from_numpy(qf).to(cuda_device), torch.from_numpy(rf).to(cuda_device)),
        ms.HALF_DEVICE: (torch.from_numpy(qf).to(cuda_device).half(), torch.from_numpy(rf).to(cuda_device).half()),
        ms.U8_DEVICE: (torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)),
        ms.U8_HOST: (q, r),
        ms.FLOAT_HOST: (torch.from_numpy(qf).pin_memory(), torch.from_numpy(rf).pin_memory()),
    }
    for typ, (qq, rr) in inputs.items():
        m = torch.zeros(500, dtype=torch.int32, device=cuda_device)
        rc = ms.cublas_2nn_sift(qq, rr, typ, 500, 3000, m, 0.8, None, 1, 0, 17)
        assert rc == ms.SIFT_OK, (typ, rc)
        np.testing.assert_array_equal(m.cpu().numpy().view(np.uint32), want, err_msg=f"type {typ}")
    # host output buffer
    m_host = np.zeros(500, np.uint32)
    assert ms.cublas_2nn_sift(q, r, ms.U8_HOST, 500, 3000, m_host, 0.8) == ms.SIFT_OK
    np.testing.assert_array_equal(m_host, want)


def test_device_brute_and_cublas_2nn_f(cuda_device):
    import torch

    q, r = datagen.make_workload(300, 2000, seed=6)
    qf = torch.from_numpy(q.astype(np.float32)).to(cuda_device)
    rf = torch.from_numpy(r.astype(np.float32)).to(cuda_device)
    s = torch.zeros((300, 4), dtype=torch.float32, device=cuda_device)
    ms.device_brute(qf, rf, 300, 2000, s)
    d, i = oracle.brute_2nn_u8(q, r)
    got = s.cpu().numpy()
    np.testing.assert_array_equal(got[:, 2:].astype(np.int64), i)
    np.testing.assert_array_equal(got[:, :2].astype(np.int64), d)
    ms.cublas_2nn_f(qf, rf, 300, 2000, s)
    d, i = oracle.brute_2nn_u8(q, r, metric=1)
    got = s.cpu().numpy()
    np.testing.assert_array_equal(got[:, 2:].astype(np.int64), i)
    np.testing.assert_array_equal(got[:, :2].astype(np.int64), d)
    # host_brute: host arrays in, host array out
    out = np.zeros((300, 4), np.float32)
    ms.host_brute(q.astype(np.float32), r.astype(np.float32), 300, 2000, out)
    d, i = oracle.brute_2nn_u8(q, r)
    np.testing.assert_array_equal(out[:, 2:].astype(np.int64), i)


def test_against_reference_gpu_functions(cuda_device):
    """The reference's own device_brute and cublas_2nn_f (built from its sources)."""
    import torch

    if not oracle.ref_available():
        pytest.skip("reference library not built")
    ref = oracle.ref()
    q, r = datagen.make_workload(400, 6000, seed=9)
    qf = torch.from_numpy(q.astype(np.float32)).to(cuda_device)
    rf = torch.from_numpy(r.astype(np.float32)).to(cuda_device)
    s_ref = torch.zeros((400, 4), dtype=torch.float32, device=cuda_device)
    s_new = torch.zeros((400, 4), dtype=torch.float32, device=cuda_device)
    assert ref.ref_device_brute(qf.data_ptr(), rf.data_ptr(), 400, 6000, s_ref.data_ptr()) == 0
    ms.device_brute(qf, rf, 400, 6000, s_new)
    a, b = s_ref.cpu().numpy(), s_new.cpu().numpy()
    np.testing.assert_array_equal(a[:, :2], b[:, :2])          # distances: exact
    same = (a[:, 2:] == b[:, 2:]).all(1)
    # index differences are allowed only where the distance ties another candidate
    d_all = ((q[~same, None, :].astype(np.int64) - r[None].astype(np.int64)) ** 2).sum(-1) if (~same).any() else None
    if d_all is not None:
        for k, row in enumerate(np.nonzero(~same)[0]):
            for c in range(2):
                assert d_all[k, int(a[row, 2 + c])] == d_all[k, int(b[row, 2 + c])]
    assert ref.ref_cublas_2nn_f(qf.data_ptr(), rf.data_ptr(), 400, 6000, s_ref.data_ptr()) == 0
    ms.cublas_2nn_f(qf, rf, 400, 6000, s_new)
    a, b = s_ref.cpu().numpy(), s_new.cpu().numpy()
    np.testing.assert_array_equal(a[:, :2], b[:, :2])


@pytest.mark.parametrize("metric", [ms.METRIC_L2, ms.METRIC_DOT])
@pytest.mark.parametrize("q_n", [700, 16_000])
def test_host_inputs_pipelined_over_base_chunks(cuda_device, kernel, metric, q_n):
    """U8_HOST with a large base: the base is copied in chunks that overlap the
    search (700 queries: chunks shrinking toward the end of the base, the copy
    setting the pace; 16,000 queries: equal chunks, the search setting it);
    results equal the device-input path bit for bit (ragged last chunk), and a
    query subset equals the oracle. The CTA-pair kernels (with and without
    folded norms) search the chunks; the single-CTA kernel takes the
    unchunked path."""
    q, r = datagen.make_workload(q_n, 200_003, seed=41)
    dev = _run(q, r, cuda_device, metric=metric)
    out = {"matches": np.zeros(q_n, np.uint32), "sorted": np.zeros((q_n, 4), np.float32),
           "nn_idx": np.zeros((q_n, 2), np.int32), "nn_dist": np.zeros((q_n, 2), np.float32)}
    rc = ms.lib().sift2nn_match(q.ctypes.data, r.ctypes.data, ms.U8_HOST, q_n, r.shape[0], metric, 0.8,
                                out["matches"].ctypes.data, out["sorted"].ctypes.data, out["nn_idx"].ctypes.data,
                                out["nn_dist"].ctypes.data, None)
    assert rc == ms.SIFT_OK
    for k in out:
        np.testing.assert_array_equal(out[k].view(np.int32) if k == "matches" else out[k],
                                      dev[k].view(np.int32) if k == "matches" else dev[k], err_msg=k)
    sel = np.arange(0, q_n, q_n // 100)
    d, i = oracle.brute_2nn_u8(q[sel], r, metric=metric)
    np.testing.assert_array_equal(out["nn_idx"][sel].astype(np.int64), i)
    np.testing.assert_array_equal(out["nn_dist"][sel].astype(np.int64), d)
    # the reference-named call on host buffers takes the same path
    m = np.zeros(q_n, np.uint32)
    if metric == ms.METRIC_L2:
        assert ms.cublas_2nn_sift(q, r, ms.U8_HOST, q_n, r.shape[0], m, 0.8) == ms.SIFT_OK
        np.testing.assert_array_equal(m, out["matches"])
