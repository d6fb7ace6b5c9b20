"""The C ABI library loads and exports what include/sift2nn.h declares (CPU only, no compute)."""
import ctypes
import os
import re

import pytest

import matching_sift_b200 as ms
from matching_sift_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# Mangled C++ forwarders that callers compiled against the reference headers
# (include/knn_brute.h) resolve to.
MANGLED = [
    "_Z15cublas_2nn_siftPvS_ijjPjfP13cublasContextimi",
    "_Z12cublas_2nn_fPA128_fS0_iiP6float4P13cublasContext",
    "_Z12device_brutePA128_fS0_iiP6float4",
    "_Z10host_brutePA128_fS0_iiP6float4",
]


def _declared_symbols():
    names = []
    for hdr in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not hdr.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", hdr)).read()
        names += re.findall(r"SIFT_API\s+[\w\s\*]+?\b(\w+)\s*\(", text)
    return names


def test_library_loads():
    lib = _native.lib()
    assert os.path.exists(_native.LIB_PATH)
    assert ms.version().startswith("sift2nn-b200")
    assert isinstance(lib, ctypes.CDLL)


def test_every_declared_symbol_is_exported():
    names = _declared_symbols()
    assert len(names) >= 9
    lib = ctypes.CDLL(_native.LIB_PATH)
    for n in names:
        assert hasattr(lib, n), n


def test_reference_mangled_symbols_are_exported():
    lib = ctypes.CDLL(_native.LIB_PATH)
    for n in MANGLED:
        assert hasattr(lib, n), n


def test_status_strings():
    for code in (0, -1, -2, -3, -4, -5, -6, -7):
        assert ms.status_string(code) != "unknown status"
    assert ms.status_string(-99) == "unknown status"


def test_no_device_is_reported_not_hidden():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import numpy as np

    q = np.zeros((4, 128), np.uint8)
    m = np.zeros(4, np.uint32)
    rc = ms.cublas_2nn_sift(q, q, ms.U8_HOST, 4, 4, m, 0.8)
    assert rc == ms.SIFT_ERR_NO_DEVICE
    with pytest.raises(ms.SiftError):
        ms.host_brute(q.astype(np.float32), q.astype(np.float32), 4, 4, np.zeros((4, 4), np.float32))
