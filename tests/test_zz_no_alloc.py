"""The zero-allocation entry point sift2nn_match_noalloc, through the C ABI.

It serves callers that cannot allocate device memory at call time (memory
owned by a custom allocator or pool, real-time loops, fixed memory budgets):
all of its scratch is a fixed __device__ array inside the library. Its results
must equal those of the allocating entry point sift2nn_match bit for bit
(exact integer search, tolerance zero), on two calls in a row, since the
second call reuses the scratch the first one left behind; at the documented
maximum sizes (16,384 x 1,048,576) a query subset is also checked against the
oracle. This file is named so that pytest collects it last.
"""
import numpy as np
import pytest

import matching_sift_b200 as ms
import oracle
from matching_sift_b200 import datagen

pytestmark = pytest.mark.gpu
MAX_Q, MAX_R = 16384, 1 << 20


def _alloc_reference(qt, rt, threshold):
    return ms.match(qt, rt, threshold=threshold, outputs=("matches", "nn_idx", "nn_dist"))


def _noalloc(lib, qt, rt, q_n, r_n, dev, stream, threshold=0.8):
    import torch

    m = torch.full((q_n,), -7, dtype=torch.int32, device=dev)
    idx = torch.full((q_n, 2), -7, dtype=torch.int32, device=dev)
    dist = torch.full((q_n, 2), -7.0, dtype=torch.float32, device=dev)
    rc = lib.sift2nn_match_noalloc(qt.data_ptr(), rt.data_ptr() if r_n else None, q_n, r_n, threshold, m.data_ptr(),
                                   idx.data_ptr(), dist.data_ptr(), stream.cuda_stream)
    return rc, m, idx, dist


def _check_equal(got, want, call):
    _, m, idx, dist = got
    np.testing.assert_array_equal(m.cpu().numpy(), want["matches"].view(np.int32), err_msg=f"call {call}")
    np.testing.assert_array_equal(idx.cpu().numpy(), want["nn_idx"], err_msg=f"call {call}")
    np.testing.assert_array_equal(dist.cpu().numpy(), want["nn_dist"], err_msg=f"call {call}")


def test_noalloc_matches_allocating_entry_point_twice(cuda_device):
    import torch

    lib = ms.lib()
    for q_n, r_n, seed in [(1000, 10000, 3), (129, 4097, 4)]:
        q, r = datagen.make_workload(q_n, r_n, seed=seed)
        qt = torch.from_numpy(q).to(cuda_device)
        rt = torch.from_numpy(r).to(cuda_device)
        want = {k: v.cpu().numpy() for k, v in _alloc_reference(qt, rt, 0.8).items()}
        stream = torch.cuda.current_stream(cuda_device)
        for call in range(2):
            got = _noalloc(lib, qt, rt, q_n, r_n, cuda_device, stream)
            assert got[0] == ms.SIFT_OK, (call, got[0])
            torch.cuda.synchronize(cuda_device)
            _check_equal(got, want, call)
        assert lib.sift2nn_noalloc_status(stream.cuda_stream) == ms.SIFT_OK


def test_noalloc_at_its_maximum_sizes(cuda_device):
    """The largest call the header promises fits the array: equal to
    sift2nn_match on two calls, a query subset equal to the oracle."""
    import torch

    lib = ms.lib()
    q, r = datagen.make_workload(MAX_Q, MAX_R, seed=5)
    qt = torch.from_numpy(q).to(cuda_device)
    rt = torch.from_numpy(r).to(cuda_device)
    want = {k: v.cpu().numpy() for k, v in _alloc_reference(qt, rt, 0.8).items()}
    stream = torch.cuda.current_stream(cuda_device)
    for call in range(2):
        got = _noalloc(lib, qt, rt, MAX_Q, MAX_R, cuda_device, stream)
        assert got[0] == ms.SIFT_OK, (call, got[0])
        torch.cuda.synchronize(cuda_device)
        _check_equal(got, want, call)
    sel = np.arange(0, MAX_Q, 256)
    d, i = oracle.brute_2nn_u8(q[sel], r)
    np.testing.assert_array_equal(got[2].cpu().numpy()[sel].astype(np.int64), i)
    np.testing.assert_array_equal(got[3].cpu().numpy()[sel].astype(np.int64), d)
    assert lib.sift2nn_noalloc_status(stream.cuda_stream) == ms.SIFT_OK


def test_noalloc_empty_base_and_no_allocation(cuda_device):
    """r_n = 0 gives "no neighbour" rows; calls change neither the device's
    free memory nor torch's allocations."""
    import torch

    lib = ms.lib()
    stream = torch.cuda.current_stream(cuda_device)
    q, r = datagen.make_workload(300, 2000, seed=6)
    qt = torch.from_numpy(q).to(cuda_device)
    rt = torch.from_numpy(r).to(cuda_device)
    rc, m, idx, dist = _noalloc(lib, qt, rt, 300, 0, cuda_device, stream)
    assert rc == ms.SIFT_OK
    torch.cuda.synchronize(cuda_device)
    assert (m.cpu().numpy().view(np.uint32) == 0xFFFFFFFF).all()
    assert (idx.cpu().numpy() == -1).all()
    assert (dist.cpu().numpy() == np.finfo(np.float32).max).all()
    outs = [torch.empty(300, dtype=torch.int32, device=cuda_device),
            torch.empty((300, 2), dtype=torch.int32, device=cuda_device),
            torch.empty((300, 2), dtype=torch.float32, device=cuda_device)]

    def call():
        return lib.sift2nn_match_noalloc(qt.data_ptr(), rt.data_ptr(), 300, 2000, 0.8, outs[0].data_ptr(),
                                         outs[1].data_ptr(), outs[2].data_ptr(), stream.cuda_stream)

    assert call() == ms.SIFT_OK and call() == ms.SIFT_OK
    torch.cuda.synchronize(cuda_device)
    free0, alloc0 = torch.cuda.mem_get_info(cuda_device)[0], torch.cuda.memory_allocated(cuda_device)
    for _ in range(3):
        assert call() == ms.SIFT_OK
    torch.cuda.synchronize(cuda_device)
    assert torch.cuda.mem_get_info(cuda_device)[0] == free0
    assert torch.cuda.memory_allocated(cuda_device) == alloc0


def test_noalloc_reports_an_expired_wait(cuda_device):
    """An expired bounded wait (the library's fault-injection probe, which
    records what an expired wait inside the search records) leaves that
    call's rows marked "no result" and is reported by sift2nn_noalloc_status;
    the next call is exact again."""
    import torch

    lib = ms.lib()
    stream = torch.cuda.current_stream(cuda_device)
    q, r = datagen.make_workload(500, 7000, seed=7)
    qt = torch.from_numpy(q).to(cuda_device)
    rt = torch.from_numpy(r).to(cuda_device)
    want = {k: v.cpu().numpy() for k, v in _alloc_reference(qt, rt, 0.8).items()}
    assert lib.sift_test_inject_wait_expiry(1) == ms.SIFT_OK
    rc, m, idx, dist = _noalloc(lib, qt, rt, 500, 7000, cuda_device, stream)
    assert rc == ms.SIFT_OK
    assert lib.sift2nn_noalloc_status(stream.cuda_stream) == ms.SIFT_ERR_DEVICE_TIMEOUT
    assert lib.sift2nn_noalloc_status(stream.cuda_stream) == ms.SIFT_OK
    assert (m.cpu().numpy().view(np.uint32) == 0xFFFFFFFF).all()
    assert (idx.cpu().numpy() == -1).all()
    assert (dist.cpu().numpy() == np.finfo(np.float32).max).all()
    got = _noalloc(lib, qt, rt, 500, 7000, cuda_device, stream)
    assert got[0] == ms.SIFT_OK
    torch.cuda.synchronize(cuda_device)
    _check_equal(got, want, "after")
    assert lib.sift2nn_noalloc_status(stream.cuda_stream) == ms.SIFT_OK


def test_noalloc_rejects_sizes_beyond_its_scratch_and_host_pointers(cuda_device):
    import torch

    lib = ms.lib()
    q = torch.zeros((16, 128), dtype=torch.uint8, device=cuda_device)
    assert lib.sift2nn_match_noalloc(q.data_ptr(), q.data_ptr(), MAX_Q + 1, 16, 0.8, None, None, None, None) == \
        ms.SIFT_ERR_INVALID_ARG
    assert lib.sift2nn_match_noalloc(q.data_ptr(), q.data_ptr(), 16, MAX_R + 1, 0.8, None, None, None, None) == \
        ms.SIFT_ERR_INVALID_ARG
    host = np.zeros((16, 128), np.uint8)
    m_host = np.zeros(16, np.uint32)
    assert lib.sift2nn_match_noalloc(host.ctypes.data, q.data_ptr(), 16, 16, 0.8, None, None, None, None) == \
        ms.SIFT_ERR_INVALID_ARG
    assert lib.sift2nn_match_noalloc(q.data_ptr(), host.ctypes.data, 16, 16, 0.8, None, None, None, None) == \
        ms.SIFT_ERR_INVALID_ARG
    assert lib.sift2nn_match_noalloc(q.data_ptr(), q.data_ptr(), 16, 16, 0.8, m_host.ctypes.data, None, None,
                                     None) == ms.SIFT_ERR_INVALID_ARG
