"""CPU oracle for the 2-NN SIFT matching path (test infrastructure only).

This package is the checker the CUDA product is compared against. Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline and
reference legs may import it; the product package never does.

Two checkers live here:

* ``liboracle.so`` (``sift_oracle.c``): a C restatement of the reference
  algorithms -- ``host_brute`` (src/knn_brute.cu:801-835), the ``-2 q.r``
  ranking of ``cublas_2nn_brute_f`` (src/knn_brute.cu:579-606), the ratio test
  of ``find_matches`` (src/knn_brute.cu:430-442) and the LSH bucketing of
  ``set_bit_h`` / ``lsh_thread_sort_reduce`` (src/lsh_h.cu:265-317, :565-629).
* ``_ref/libref.so``: the reference implementation compiled unmodified from its
  own sources (``make -C oracle ref``), re-exported with C linkage by
  ``ref_shim.cu``. Its ``host_brute`` pins the restatement (golden fixtures in
  ``tests/golden``) and is the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "liboracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libref.so")
_CALLER = os.path.join(_HERE, "_ref", "reference_caller")


def _reference_dir() -> str:
    """Where the reference checkout lives: $SIFT_REFERENCE_DIR, else the path in
    oracle/reference_dir.txt (configuration of the build machine), else ''."""
    env = os.environ.get("SIFT_REFERENCE_DIR")
    if env:
        return env
    cfg = os.path.join(_HERE, "reference_dir.txt")
    if os.path.exists(cfg):
        with open(cfg) as f:
            return f.read().strip()
    return ""


REF_SRC = _reference_dir()

_lib = None
_ref = None

_i64p = ctypes.POINTER(ctypes.c_int64)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def build(force: bool = False) -> None:
    """Compile liboracle.so (gcc) and, when the reference sources exist, _ref/libref.so (nvcc)."""
    if force or not os.path.exists(_ORACLE_SO):
        subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)
    if REF_SRC and os.path.isdir(os.path.join(REF_SRC, "src")) and (
            force or not os.path.exists(_REF_SO) or not os.path.exists(_CALLER)):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF={REF_SRC}"], check=True)


def reference_caller() -> str:
    """Path of the C++ program that calls the library through the reference's own headers ('' if not built)."""
    return _CALLER if os.path.exists(_CALLER) else ""


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_ORACLE_SO):
            build()
        _lib = ctypes.CDLL(_ORACLE_SO)
        _lib.oracle_2nn_u8.restype = ctypes.c_int
        _lib.oracle_2nn_u8.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        _lib.oracle_2nn_f64.restype = ctypes.c_int
        _lib.oracle_2nn_f64.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        _lib.oracle_ratio_match.restype = None
        _lib.oracle_ratio_match.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_float,
                                            ctypes.c_void_p]
        _lib.oracle_lsh_codes.restype = None
        _lib.oracle_lsh_codes.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_void_p]
        _lib.oracle_bucket_sort.restype = ctypes.c_int64
        _lib.oracle_bucket_sort.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_void_p, ctypes.c_void_p]
        _lib.oracle_lsh_scan.restype = ctypes.c_int
        _lib.oracle_lsh_scan.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p]
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF_SO)


def ref():
    """The reference implementation built from its own sources (checker / CPU baseline)."""
    global _ref
    if _ref is None:
        if not os.path.exists(_REF_SO):
            raise FileNotFoundError(f"{_REF_SO} missing: run `make -C oracle ref` where the reference sources exist")
        _ref = ctypes.CDLL(_REF_SO)
        _ref.ref_host_brute_mt.restype = None
        _ref.ref_host_brute_mt.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_void_p, ctypes.c_int]
        for name in ("ref_device_brute", "ref_cublas_2nn_f"):
            f = getattr(_ref, name)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        _ref.ref_cublas_2nn_sift.restype = ctypes.c_int
        _ref.ref_cublas_2nn_sift.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32,
                                             ctypes.c_void_p, ctypes.c_float, ctypes.c_int, ctypes.c_size_t,
                                             ctypes.c_int]
        _ref.ref_lsh_buckets.restype = ctypes.c_int
        _ref.ref_lsh_buckets.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return _ref


def _ptr(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


# ------------------------------------------------------------------ 2-NN ---

def brute_2nn_u8(q: np.ndarray, r: np.ndarray, metric: int = 0, nthreads: int | None = None):
    """Exact lexicographic 2-NN (restates host_brute). Returns (dist[q,2] int64, idx[q,2] int64).

    metric 0: full squared L2; metric 1: -2 q.r (the cublas_2nn_f ranking).
    Absent neighbours: dist INT64_MAX, idx -1.
    """
    q = np.ascontiguousarray(q, dtype=np.uint8)
    r = np.ascontiguousarray(r, dtype=np.uint8)
    assert q.ndim == 2 and q.shape[1] == 128 and r.ndim == 2 and r.shape[1] == 128
    d = np.empty((q.shape[0], 2), np.int64)
    i = np.empty((q.shape[0], 2), np.int64)
    nt = nthreads or os.cpu_count() or 1
    rc = lib().oracle_2nn_u8(_ptr(q), _ptr(r), q.shape[0], r.shape[0], metric, nt, _ptr(d), _ptr(i))
    if rc != 0:
        raise RuntimeError(f"oracle_2nn_u8 failed: {rc}")
    return d, i


def brute_2nn_f64(q: np.ndarray, r: np.ndarray, metric: int = 0, nthreads: int | None = None):
    """FP64 2-NN of float descriptors. Returns (dist[q,2] float64, idx[q,2] int64)."""
    q = np.ascontiguousarray(q, dtype=np.float32)
    r = np.ascontiguousarray(r, dtype=np.float32)
    d = np.empty((q.shape[0], 2), np.float64)
    i = np.empty((q.shape[0], 2), np.int64)
    nt = nthreads or os.cpu_count() or 1
    rc = lib().oracle_2nn_f64(_ptr(q), _ptr(r), q.shape[0], r.shape[0], metric, nt, _ptr(d), _ptr(i))
    if rc != 0:
        raise RuntimeError(f"oracle_2nn_f64 failed: {rc}")
    return d, i


def ratio_match(dist: np.ndarray, idx: np.ndarray, threshold: float) -> np.ndarray:
    """matches[q] = idx1 if sqrtf(d1)/sqrtf(d2) < threshold else UINT32_MAX (float32 arithmetic)."""
    dist = np.ascontiguousarray(dist, dtype=np.int64)
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    out = np.empty(dist.shape[0], np.uint32)
    lib().oracle_ratio_match(_ptr(dist), _ptr(idx), dist.shape[0], threshold, _ptr(out))
    return out


def mutual_match(a: np.ndarray, b: np.ndarray, threshold: float) -> np.ndarray:
    """Mutual nearest neighbours of two descriptor sets (cross-check; no
    counterpart in the reference, composed from brute_2nn_u8 in both
    directions): out[i] = j when j is the nearest row of b for row i of a,
    row i is the nearest row of a for row j of b and, when threshold > 0, the
    ratio test of row i passes; else UINT32_MAX."""
    d, i = brute_2nn_u8(a, b)
    out = np.full(a.shape[0], 0xFFFFFFFF, np.uint32)
    if a.shape[0] == 0 or b.shape[0] == 0:
        return out
    _, ir = brute_2nn_u8(b, a)
    j = i[:, 0]
    ok = j >= 0
    if threshold > 0:
        ok &= ratio_match(d, i, threshold) != 0xFFFFFFFF
    back = np.where(ok, ir[np.where(ok, j, 0), 0], -1)
    keep = ok & (back == np.arange(a.shape[0]))
    out[keep] = j[keep].astype(np.uint32)
    return out


# ------------------------------------------------------------------- LSH ---

def lsh_codes(x: np.ndarray, planes: np.ndarray):
    """Sign-bit codes (bit j set when x.h_j < 0) with FP64 dots. Returns (codes uint32, dots float64)."""
    x = np.ascontiguousarray(x, dtype=np.uint8)
    planes = np.ascontiguousarray(planes, dtype=np.float32)
    nbits = planes.shape[0]
    code = np.empty(x.shape[0], np.uint32)
    dots = np.empty((x.shape[0], nbits), np.float64)
    lib().oracle_lsh_codes(_ptr(x), x.shape[0], _ptr(planes), nbits, _ptr(code), _ptr(dots))
    return code, dots


def bucket_sort(code: np.ndarray):
    """(order, bucket_code, bucket_start, bucket_count) grouping points by code, ties by id."""
    code = np.ascontiguousarray(code, dtype=np.uint32)
    n = code.shape[0]
    order = np.empty(max(n, 1), np.int64)
    bc = np.empty(max(n, 1), np.uint32)
    bs = np.empty(max(n, 1), np.int64)
    bn = np.empty(max(n, 1), np.int64)
    nb = lib().oracle_bucket_sort(_ptr(code), n, _ptr(order), _ptr(bc), _ptr(bs), _ptr(bn))
    return order[:n], bc[:nb], bs[:nb], bn[:nb]


def lsh_scan(q: np.ndarray, r: np.ndarray, q_codes: np.ndarray, r_codes: np.ndarray):
    """Exact 2-NN of each query over the union of its buckets in all L tables.

    q_codes: [L, q_n] uint32, r_codes: [L, r_n] uint32. Returns (dist int64 [q,2], idx int64 [q,2]).
    """
    q = np.ascontiguousarray(q, dtype=np.uint8)
    r = np.ascontiguousarray(r, dtype=np.uint8)
    q_codes = np.ascontiguousarray(q_codes, dtype=np.uint32)
    r_codes = np.ascontiguousarray(r_codes, dtype=np.uint32)
    L = q_codes.shape[0]
    d = np.empty((q.shape[0], 2), np.int64)
    i = np.empty((q.shape[0], 2), np.int64)
    rc = lib().oracle_lsh_scan(_ptr(q), q.shape[0], _ptr(r), r.shape[0], _ptr(q_codes), _ptr(r_codes), L,
                               _ptr(d), _ptr(i))
    if rc != 0:
        raise RuntimeError("oracle_lsh_scan failed")
    return d, i


# ----------------------------------------------------- reference library ---

def ref_host_brute(q: np.ndarray, r: np.ndarray, nthreads: int = 1) -> np.ndarray:
    """The reference host_brute (compiled from its sources) -> float4 rows {d1, d2, i1, i2}."""
    q = np.ascontiguousarray(q, dtype=np.float32)
    r = np.ascontiguousarray(r, dtype=np.float32)
    out = np.empty((q.shape[0], 4), np.float32)
    ref().ref_host_brute_mt(_ptr(q), _ptr(r), q.shape[0], r.shape[0], _ptr(out), nthreads)
    return out
