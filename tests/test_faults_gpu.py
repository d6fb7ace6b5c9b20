"""Failure detection without a GPU fault, and GPU-side ordering of calls on
different streams, through the C ABI.

* An expired bounded wait: the library's probe waits on an mbarrier that
  nothing completes (the bounded wait every pipeline stage of the search
  kernels uses), gives up after 1 ms and records the device error the host
  reads back; the context stays usable and the next search is bit-exact.
* A failed scratch allocation (injected on the host) is reported as
  SIFT_ERR_ALLOC and the next call succeeds.
* Two searches issued on two streams share the scratch arena; the library
  orders them on the GPU, so both equal the oracle.
The reference checks no error at all (src/knn_brute.cu:254-275).
"""
import numpy as np
import pytest

import matching_sift_b200 as ms
import oracle
from matching_sift_b200 import datagen

pytestmark = pytest.mark.gpu


def _search(qt, rt):
    out = ms.match(qt, rt, threshold=0.8, outputs=("matches", "nn_idx", "nn_dist"))
    return out


def test_expired_wait_is_reported_and_the_context_recovers(cuda_device):
    import torch

    q, r = datagen.make_workload(300, 5000, seed=51)
    qt, rt = torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)
    assert ms.stream_status() == ms.SIFT_OK
    assert ms.lib().sift_test_inject_wait_expiry(1) == ms.SIFT_OK
    _search(qt, rt)
    assert ms.stream_status() == ms.SIFT_ERR_DEVICE_TIMEOUT
    assert ms.stream_status() == ms.SIFT_OK          # read and cleared
    out = _search(qt, rt)
    assert ms.stream_status() == ms.SIFT_OK
    d, i = oracle.brute_2nn_u8(q, r)
    np.testing.assert_array_equal(out["nn_idx"].cpu().numpy().astype(np.int64), i)
    np.testing.assert_array_equal(out["nn_dist"].cpu().numpy().astype(np.int64), d)
    # a synchronous reference-named entry point reports it as its return value
    assert ms.lib().sift_test_inject_wait_expiry(1) == ms.SIFT_OK
    m = torch.zeros(300, dtype=torch.int32, device=cuda_device)
    assert ms.cublas_2nn_sift(qt, rt, ms.U8_DEVICE, 300, 5000, m, 0.8) == ms.SIFT_ERR_DEVICE_TIMEOUT
    assert ms.cublas_2nn_sift(qt, rt, ms.U8_DEVICE, 300, 5000, m, 0.8) == ms.SIFT_OK
    np.testing.assert_array_equal(m.cpu().numpy().view(np.uint32), oracle.ratio_match(d, i, 0.8))


def test_failed_scratch_allocation_is_reported(cuda_device):
    import torch

    q, r = datagen.make_workload(200, 3000, seed=52)
    qt, rt = torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device)
    assert ms.lib().sift_test_fail_arena(1) == ms.SIFT_OK
    with pytest.raises(ms.SiftError) as e:
        _search(qt, rt)
    assert e.value.status == ms.SIFT_ERR_ALLOC
    out = _search(qt, rt)
    assert ms.stream_status() == ms.SIFT_OK
    d, i = oracle.brute_2nn_u8(q, r)
    np.testing.assert_array_equal(out["nn_idx"].cpu().numpy().astype(np.int64), i)
    assert ms.lib().sift_test_fail_arena(-1) == ms.SIFT_ERR_INVALID_ARG
    assert ms.lib().sift_test_inject_wait_expiry(-1) == ms.SIFT_ERR_INVALID_ARG


def test_calls_on_two_streams_do_not_share_scratch_at_once(cuda_device):
    """Each call's kernels wait for the previous call's on the GPU, whatever
    stream it used: two large searches enqueued back to back on two streams
    both equal the oracle."""
    import torch

    qa, ra = datagen.make_workload(4000, 60000, seed=53)
    qb, rb = datagen.make_workload(3000, 80000, seed=54)
    ta = [torch.from_numpy(x).to(cuda_device) for x in (qa, ra)]
    tb = [torch.from_numpy(x).to(cuda_device) for x in (qb, rb)]
    sa, sb = torch.cuda.Stream(cuda_device), torch.cuda.Stream(cuda_device)
    torch.cuda.synchronize(cuda_device)
    for _ in range(3):
        oa = ms.match(*ta, threshold=0.8, stream=sa, outputs=("nn_idx", "nn_dist"))
        ob = ms.match(*tb, threshold=0.8, stream=sb, outputs=("nn_idx", "nn_dist"))
        torch.cuda.synchronize(cuda_device)
        assert ms.stream_status() == ms.SIFT_OK
        for (q, r), o in (((qa, ra), oa), ((qb, rb), ob)):
            sel = np.arange(0, q.shape[0], 5)
            d, i = oracle.brute_2nn_u8(q[sel], r)
            np.testing.assert_array_equal(o["nn_idx"].cpu().numpy()[sel].astype(np.int64), i)
            np.testing.assert_array_equal(o["nn_dist"].cpu().numpy()[sel].astype(np.int64), d)
