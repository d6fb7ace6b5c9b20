"""Loader for libsift2nn.so, the CUDA product library (sm_100a).

There is no CPU path: if the library is missing this module raises, and every
compute call on a machine without a usable B200 returns SIFT_ERR_NO_DEVICE.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsift2nn.so")

SIFT_OK = 0
SIFT_ERR_INVALID_ARG = -1
SIFT_ERR_CUDA = -2
SIFT_ERR_NOT_INTEGER = -3
SIFT_ERR_DEVICE_TIMEOUT = -4
SIFT_ERR_NO_DEVICE = -5
SIFT_ERR_UNSUPPORTED = -6
SIFT_ERR_ALLOC = -7

FLOAT_HOST, FLOAT_DEVICE, HALF_DEVICE, U8_DEVICE, U8_HOST = 0, 1, 2, 3, 4
METRIC_L2, METRIC_DOT = 0, 1

_vp = ctypes.c_void_p
_PROTOS = {
    "cublas_2nn_sift": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, _vp,
                                       ctypes.c_float, _vp, ctypes.c_int, ctypes.c_size_t, ctypes.c_int]),
    "cublas_2nn_f": (None, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "device_brute": (None, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "host_brute": (None, [_vp, _vp, ctypes.c_int, ctypes.c_int, _vp]),
    "sift_last_status": (ctypes.c_int, []),
    "sift2nn_match": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                     ctypes.c_float, _vp, _vp, _vp, _vp, _vp]),
    "sift_stream_status": (ctypes.c_int, [_vp]),
    "sift_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "sift_version": (ctypes.c_char_p, []),
    "sift_launch_count": (ctypes.c_longlong, []),
    "sift_profile_enable": (None, [ctypes.c_int]),
    "sift_profile_collect": (ctypes.c_int, [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]),
    "sift_profile_collect_kernel": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                                   ctypes.POINTER(ctypes.c_int)]),
    "sift_set_kernel_variant": (ctypes.c_int, [ctypes.c_int]),
    "lsh_gpu": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, _vp, ctypes.c_float, _vp,
                               ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "sift_lsh_hash": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, ctypes.c_int, ctypes.c_int, _vp, _vp]),
    "sift_lsh_buckets": (ctypes.c_int, [_vp, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "sift_lsh_match_probes": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, _vp,
                                             ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, _vp, _vp, _vp,
                                             _vp, _vp]),
    "sift_lsh_match": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, _vp, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_float, _vp, _vp, _vp, _vp]),
    "sift2nn_match_noalloc": (ctypes.c_int, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float, _vp, _vp,
                                             _vp, _vp]),
    "sift2nn_noalloc_status": (ctypes.c_int, [_vp]),
    "sift_test_inject_wait_expiry": (ctypes.c_int, [ctypes.c_int]),
    "sift_test_fail_arena": (ctypes.c_int, [ctypes.c_int]),
    "sift2nn_match_batch": (ctypes.c_int, [_vp, _vp, ctypes.c_uint32, _vp, ctypes.c_int, ctypes.c_float, _vp, _vp,
                                           _vp, _vp]),
    "sift_merge_top2": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_float, _vp, _vp, _vp,
                                       _vp]),
    "sift_compact_matches": (ctypes.c_int, [_vp, _vp, ctypes.c_uint32, _vp, ctypes.c_int, _vp, ctypes.c_uint32, _vp,
                                            _vp]),
    "sift2nn_match_mutual_batch": (ctypes.c_int, [_vp, _vp, ctypes.c_uint32, _vp, ctypes.c_int, ctypes.c_float, _vp,
                                                  _vp, _vp, _vp]),
    "sift_batch_plan_create": (ctypes.c_int, [_vp, _vp, ctypes.c_uint32, _vp, ctypes.c_int, ctypes.c_float, _vp, _vp,
                                              _vp, ctypes.c_int, ctypes.POINTER(_vp)]),
    "sift_batch_plan_run": (ctypes.c_int, [_vp, _vp]),
    "sift_batch_plan_info": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_float)]),
    "sift_batch_plan_destroy": (None, [_vp]),
    "sift_batch_describe": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_longlong)]),
    "sift_mlp_train": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, ctypes.c_uint32, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                      ctypes.c_ulonglong, _vp, _vp, _vp, _vp, _vp, _vp]),
    "sift_mlp_hash": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, _vp, _vp, _vp]),
    "sift_mlp_match": (ctypes.c_int, [_vp, _vp, ctypes.c_uint32, ctypes.c_uint32, _vp, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_float, ctypes.c_float, _vp, _vp, _vp, _vp,
                                      ctypes.POINTER(ctypes.c_uint32), _vp]),
    "sift_lsh_index_create": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, ctypes.c_int, ctypes.c_int,
                                             ctypes.POINTER(_vp)]),
    "sift_mlp_index_create": (ctypes.c_int, [_vp, ctypes.c_uint32, _vp, ctypes.POINTER(_vp)]),
    "sift_index_search": (ctypes.c_int, [_vp, _vp, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                         ctypes.c_float, _vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_uint32), _vp]),
    "sift_index_buckets": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_int), _vp]),
    "sift_index_destroy": (None, [_vp]),
    "sift_mlp_loss_grad": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, ctypes.c_float, ctypes.c_float, _vp,
                                          ctypes.POINTER(ctypes.c_float)]),
}


class sift_mlp(ctypes.Structure):
    """C layout of `sift_mlp` (include/sift2nn.h)."""
    _fields_ = [("w1", ctypes.c_void_p), ("b1", ctypes.c_void_p), ("w2", ctypes.c_void_p),
                ("b2", ctypes.c_void_p), ("k", ctypes.c_int)]


SIFT_MLP_PARAMS = 256 * 128 + 256 + 32 * 256 + 32

SIFT_BATCH_TUNE = 1


def SIFT_BATCH_SHAPE(k: int) -> int:
    return (k + 1) << 4

_lib = None


class SiftError(RuntimeError):
    def __init__(self, status: int, where: str = ""):
        self.status = status
        msg = status_string(status) if _lib is not None else str(status)
        super().__init__(f"{where}: {msg} ({status})" if where else f"{msg} ({status})")


def lib() -> ctypes.CDLL:
    """The loaded product library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C matching_sift_b200` "
                              "(or __graft_entry__.build()); there is no CPU fallback")
        so = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            f = getattr(so, name)
            f.restype = res
            f.argtypes = args
        _lib = so
    return _lib


def status_string(status: int) -> str:
    return lib().sift_status_string(status).decode()


def check(status: int, where: str = "") -> None:
    if status != SIFT_OK:
        raise SiftError(status, where)
