"""A C++ program compiled against the reference's own headers
(include/knn_brute.h, include/lsh_h.h) and linked to libsift2nn.so calls
cublas_2nn_sift, cublas_2nn_f, device_brute, host_brute and lsh_gpu by their
mangled C++ names (tests/cxx/reference_caller.cu, built into oracle/_ref by
`make -C oracle ref`). Its outputs -- float4 rows passed through the
reference's own `float4*` / `des_t_f*` types -- are checked against the oracle
and against the C ABI."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import matching_sift_b200 as ms
import oracle
from matching_sift_b200 import datagen

MANGLED = ["_Z15cublas_2nn_siftPvS_ijjPjfP13cublasContextimi", "_Z12cublas_2nn_fPA128_fS0_iiP6float4P13cublasContext",
           "_Z12device_brutePA128_fS0_iiP6float4", "_Z10host_brutePA128_fS0_iiP6float4",
           "_Z7lsh_gpuPvS_ijjPjfP13cublasContextiiii"]
FLT_MAX = np.float32(np.finfo(np.float32).max)


def _caller():
    path = oracle.reference_caller()
    if not path:
        pytest.skip("reference caller not built (needs the reference headers at build time)")
    return path


def test_caller_resolves_the_mangled_entry_points():
    """The program's undefined reference symbols are exactly the library's forwarders (no GPU needed)."""
    path = _caller()
    und = subprocess.run(["nm", "-D", "-u", path], check=True, capture_output=True, text=True).stdout
    wanted = [name for name in MANGLED if name in und]
    assert wanted == MANGLED
    lib = ctypes.CDLL(ms.LIB_PATH)
    for name in MANGLED:
        assert hasattr(lib, name), name


@pytest.mark.gpu
def test_cxx_caller_outputs(cuda_device, tmp_path):
    path = _caller()
    q_n, r_n = 500, 9000
    q, r = datagen.make_workload(q_n, r_n, seed=61)
    q.astype(np.float32).tofile(tmp_path / "q.f32")
    r.astype(np.float32).tofile(tmp_path / "r.f32")
    res = subprocess.run([path, str(tmp_path), str(q_n), str(r_n)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    rc_sift, rc_lsh = map(int, (tmp_path / "status.txt").read_text().split())
    assert rc_sift == ms.SIFT_OK and rc_lsh == ms.SIFT_OK

    d, i = oracle.brute_2nn_u8(q, r)
    np.testing.assert_array_equal(np.fromfile(tmp_path / "sift.u32", np.uint32), oracle.ratio_match(d, i, 0.8))
    want = np.concatenate([d.astype(np.float32), i.astype(np.float32)], axis=1)
    for name in ("device_brute", "host_brute"):
        got = np.fromfile(tmp_path / f"{name}.f32", np.float32).reshape(q_n, 4)
        np.testing.assert_array_equal(got, want, err_msg=name)
    dd, di = oracle.brute_2nn_u8(q, r, metric=1)
    got = np.fromfile(tmp_path / "f.f32", np.float32).reshape(q_n, 4)
    np.testing.assert_array_equal(got, np.concatenate([dd.astype(np.float32), di.astype(np.float32)], axis=1))

    # lsh_gpu: the +/-1 planes the program's srand(1234) + rand() produce, in
    # the reference's draw order, given to the native LSH call.
    import torch

    libc = ctypes.CDLL("libc.so.6")
    libc.srand(1234)
    L, nbits = 3, 10
    planes = np.empty((L, nbits, 128), np.int8)
    rand_max = np.float32(2147483647)
    for t in range(L):
        for j in range(nbits):
            for c in range(128):
                planes[t, j, c] = 1 if float(np.float32(libc.rand()) / rand_max) - 0.5 >= 0 else -1
    want = ms.lsh_match(torch.from_numpy(q).to(cuda_device), torch.from_numpy(r).to(cuda_device),
                        torch.from_numpy(planes).to(cuda_device), threshold=0.0)["matches"].cpu().numpy()
    np.testing.assert_array_equal(np.fromfile(tmp_path / "lsh.u32", np.uint32), want.view(np.uint32))
