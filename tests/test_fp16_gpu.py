"""FP16 tensor-core kernel and power-of-two scaled inputs, through the C ABI.

Half rows (SIFT_HALF_DEVICE) are searched in place by the kind::f16 kernel
with f32 accumulation. Their values are integers in [0, 255] times 2^-s, so
every dot product is exact and the results must equal the oracle's bit for
bit, distances in the caller's units (integer distance x 2^-2s). The same
holds for float inputs, packed to u8 after the common scale is found; the
reference's own benchmark feeds SIFT components / 512 (src/test.cu:99-103).
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


def _run(q, r, dev, dtype, scale=1.0, metric=ms.METRIC_L2, threshold=0.8):
    import torch

    qt = (torch.from_numpy(np.ascontiguousarray(q)).to(dev).to(torch.float32) * scale).to(dtype)
    rt = (torch.from_numpy(np.ascontiguousarray(r)).to(dev).to(torch.float32) * scale).to(dtype)
    out = ms.match(qt, rt, threshold=threshold, metric=metric, outputs=("matches", "nn_idx", "nn_dist", "sorted"))
    assert ms.stream_status() == ms.SIFT_OK
    return {k: v.cpu().numpy() for k, v in out.items()}


def _check(q, r, got, scale=1.0, metric=ms.METRIC_L2):
    d, i = oracle.brute_2nn_u8(q, r, metric=metric)
    np.testing.assert_array_equal(got["nn_idx"].astype(np.int64), i)
    present = i >= 0
    want = (d[present].astype(np.float64) * scale * scale).astype(np.float32)
    np.testing.assert_array_equal(got["nn_dist"][present], want)
    assert (got["nn_dist"][~present] == FLT_MAX).all()
    return d, i


@pytest.fixture(params=["f16_kernel", "u8_kernel"])
def half_path(request):
    """Half inputs through the FP16 kernel (variant 0) and packed to u8 (variant 2)."""
    ms.lib().sift_set_kernel_variant(0 if request.param == "f16_kernel" else 2)
    yield request.param
    ms.lib().sift_set_kernel_variant(0)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "host_brute_*.npz"))), ids=os.path.basename)
def test_fp16_golden_host_brute(cuda_device, path):
    import torch

    z = np.load(path)
    got = _run(z["q"], z["r"], cuda_device, torch.float16)
    np.testing.assert_array_equal(got["sorted"], z["sorted"])


@pytest.mark.parametrize("metric", [ms.METRIC_L2, ms.METRIC_DOT])
def test_fp16_config1_vs_oracle(cuda_device, half_path, metric):
    import torch

    q, r = datagen.make_workload(1000, 10000, seed=0)
    got = _run(q, r, cuda_device, torch.float16, metric=metric)
    d, i = _check(q, r, got, metric=metric)
    if metric == ms.METRIC_L2:
        np.testing.assert_array_equal(got["matches"], oracle.ratio_match(d, i, 0.8))


@pytest.mark.parametrize("q_n,r_n", [(1, 1), (3, 300), (127, 255), (129, 257), (255, 513), (300, 4097), (2048, 1)])
def test_fp16_ragged_sizes(cuda_device, q_n, r_n):
    import torch

    q, r = datagen.make_workload(q_n, r_n, seed=q_n * 7 + r_n)
    _check(q, r, _run(q, r, cuda_device, torch.float16))


def test_fp16_extreme_values_and_ties(cuda_device):
    import torch

    r = np.stack([np.zeros(128, np.uint8), np.full(128, 255, np.uint8)] * 200)
    q = np.stack([np.full(128, 255, np.uint8), np.zeros(128, np.uint8), np.full(128, 128, np.uint8)] * 50)
    got = _run(q, r, cuda_device, torch.float16)
    _check(q, r, got)
    assert got["nn_dist"][2, 0] == 128 * 127 ** 2


@pytest.mark.parametrize("scale", [1.0 / 512, 0.5, 2.0 ** -24])
@pytest.mark.parametrize("dtype", ["float16", "float32"])
def test_power_of_two_scaled_inputs(cuda_device, half_path, scale, dtype):
    """Integers times 2^-s give the integer results scaled by 2^-2s."""
    import torch

    q, r = datagen.make_workload(500, 3000, seed=11)
    got = _run(q, r, cuda_device, getattr(torch, dtype), scale=scale)
    d, i = _check(q, r, got, scale=scale)
    np.testing.assert_array_equal(got["matches"], oracle.ratio_match(d, i, 0.8))


def test_reference_benchmark_scaling_through_cublas_2nn_sift(cuda_device):
    """cublas_2nn_sift on components / 512 in float (FLOAT_DEVICE) and half
    (HALF_DEVICE), the reference benchmark's input convention."""
    import torch

    q, r = datagen.make_workload(400, 5000, seed=12)
    d, i = oracle.brute_2nn_u8(q, r)
    want = oracle.ratio_match(d, i, 0.8)
    for typ, dt in ((ms.FLOAT_DEVICE, torch.float32), (ms.HALF_DEVICE, torch.float16)):
        qq = (torch.from_numpy(q).to(cuda_device).float() / 512).to(dt)
        rr = (torch.from_numpy(r).to(cuda_device).float() / 512).to(dt)
        m = torch.zeros(400, dtype=torch.int32, device=cuda_device)
        assert ms.cublas_2nn_sift(qq, rr, typ, 400, 5000, m, 0.8) == ms.SIFT_OK
        np.testing.assert_array_equal(m.cpu().numpy().view(np.uint32), want)
    # device_brute on scaled floats: distances in the caller's units, exactly.
    qf = torch.from_numpy(q).to(cuda_device).float() / 512
    rf = torch.from_numpy(r).to(cuda_device).float() / 512
    s = torch.zeros((400, 4), dtype=torch.float32, device=cuda_device)
    ms.device_brute(qf, rf, 400, 5000, s)
    got = s.cpu().numpy()
    np.testing.assert_array_equal(got[:, 2:].astype(np.int64), i)
    np.testing.assert_array_equal(got[:, :2], (d.astype(np.float64) / 2 ** 18).astype(np.float32))


@pytest.mark.parametrize("bad", ["negative", "too_large", "not_dyadic"])
def test_values_outside_the_integer_contract_take_the_float_path(cuda_device, bad):
    """One value that is not an integer in [0, 255] (times a power of two)
    sends the whole search to the general float path; its results then
    agree with the FP64 oracle within the float path's tolerance."""
    import torch

    from test_float_gpu import check_2nn

    q, r = datagen.make_workload(20, 100, seed=13)
    qf = torch.from_numpy(q).to(cuda_device).float()
    qf[3, 7] = {"negative": -1.0, "too_large": 256.0, "not_dyadic": 0.1}[bad]
    rf = torch.from_numpy(r).to(cuda_device).float()
    for dt in (torch.float32, torch.float16):
        out = ms.match(qf.to(dt), rf.to(dt), outputs=("nn_idx", "nn_dist"))
        assert ms.stream_status() == ms.SIFT_OK
        check_2nn(qf.to(dt).float().cpu().numpy(), rf.to(dt).float().cpu().numpy(), out["nn_dist"].cpu().numpy(),
                  out["nn_idx"].cpu().numpy())


def test_fp16_scale_subset_vs_oracle(cuda_device):
    """10,000 x 1,000,000 half rows: 64 random queries against the oracle, and
    both distances of every query recomputed from the returned indices."""
    import torch

    q, r = datagen.make_workload(10000, 1000000, seed=0)
    got = _run(q, r, cuda_device, torch.float16)
    sel = np.sort(np.random.default_rng(2).choice(q.shape[0], 64, replace=False))
    d, i = oracle.brute_2nn_u8(q[sel], r)
    np.testing.assert_array_equal(got["nn_idx"][sel].astype(np.int64), i)
    np.testing.assert_array_equal(got["nn_dist"][sel].astype(np.int64), d)
    idx = got["nn_idx"].astype(np.int64)
    for k in range(2):
        dd = ((q.astype(np.int64) - r[idx[:, k]].astype(np.int64)) ** 2).sum(1)
        np.testing.assert_array_equal(dd, got["nn_dist"][:, k].astype(np.int64))
