"""The zero-allocation entry point sift2nn_match_noalloc, through the C ABI.

It serves callers that cannot allocate device memory at call time (memory
owned by a custom allocator or pool, real-time loops, fixed memory budgets):
all of its scratch is a fixed __device__ array inside the library. Its results
must equal those of the allocating entry point sift2nn_match bit for bit
(exact integer search, tolerance zero), on two calls in a row, since the
second call reuses the scratch the first one left behind. This file is named
so that pytest collects it last.
"""
import numpy as np
import pytest

import matching_sift_b200 as ms
from matching_sift_b200 import datagen

pytestmark = pytest.mark.gpu


def _alloc_reference(qt, rt, threshold):
    return ms.match(qt, rt, threshold=threshold, outputs=("matches", "nn_idx", "nn_dist"))


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
            m = torch.full((q_n,), -7, dtype=torch.int32, device=cuda_device)
            idx = torch.full((q_n, 2), -7, dtype=torch.int32, device=cuda_device)
            dist = torch.full((q_n, 2), -7.0, dtype=torch.float32, device=cuda_device)
            rc = lib.sift2nn_match_noalloc(qt.data_ptr(), rt.data_ptr(), q_n, r_n, 0.8, m.data_ptr(), idx.data_ptr(),
                                           dist.data_ptr(), stream.cuda_stream)
            assert rc == ms.SIFT_OK, (call, rc)
            torch.cuda.synchronize(cuda_device)
            np.testing.assert_array_equal(m.cpu().numpy(), want["matches"].view(np.int32), err_msg=f"call {call}")
            np.testing.assert_array_equal(idx.cpu().numpy(), want["nn_idx"], err_msg=f"call {call}")
            np.testing.assert_array_equal(dist.cpu().numpy(), want["nn_dist"], err_msg=f"call {call}")


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda_device):
    import torch

    lib = ms.lib()
    q = torch.zeros((16, 128), dtype=torch.uint8, device=cuda_device)
    assert lib.sift2nn_match_noalloc(q.data_ptr(), q.data_ptr(), 16385, 16, 0.8, None, None, None, None) == \
        ms.SIFT_ERR_INVALID_ARG
    assert lib.sift2nn_match_noalloc(q.data_ptr(), q.data_ptr(), 16, (1 << 20) + 1, 0.8, None, None, None, None) == \
        ms.SIFT_ERR_INVALID_ARG
