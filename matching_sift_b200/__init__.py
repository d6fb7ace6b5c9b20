"""B200-native 2-NN SIFT descriptor matching.

Host-side mirror of the reference's matching interface (src/knn_brute.cu,
src/lsh_h.cu): the functions below keep the reference's names and argument
order and call the CUDA library ``libsift2nn.so`` through its C ABI
(``include/sift2nn.h``). Pointers may be given as integers, torch tensors or
numpy arrays. Unlike the reference, failures are reported: int-returning
functions return the status, void ones raise :class:`SiftError`.

``match`` is the native convenience call on torch tensors.
"""
from __future__ import annotations

import ctypes

from ._native import (SIFT_BATCH_SHAPE, SIFT_BATCH_TUNE, SIFT_MLP_PARAMS, sift_mlp,
                      FLOAT_DEVICE, FLOAT_HOST, HALF_DEVICE, METRIC_DOT, METRIC_L2, SIFT_ERR_ALLOC,
                      SIFT_ERR_CUDA, SIFT_ERR_DEVICE_TIMEOUT, SIFT_ERR_INVALID_ARG, SIFT_ERR_NO_DEVICE,
                      SIFT_ERR_NOT_INTEGER, SIFT_ERR_UNSUPPORTED, SIFT_OK, U8_DEVICE, U8_HOST, LIB_PATH,
                      SiftError, check, lib, status_string)

__all__ = [
    "cublas_2nn_sift", "cublas_2nn_f", "device_brute", "host_brute", "lsh_gpu", "match", "lsh_match", "lsh_hash", "lsh_buckets",
    "stream_status", "version", "match_batch", "match_mutual", "match_mutual_batch", "compact_matches", "BatchPlan", "batch_describe",
    "MlpHash", "mlp_loss_grad", "HashIndex",
    "SiftError", "FLOAT_HOST", "FLOAT_DEVICE", "HALF_DEVICE", "U8_DEVICE", "U8_HOST", "METRIC_L2", "METRIC_DOT",
]


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    if hasattr(x, "ctypes"):
        return x.ctypes.data
    if isinstance(x, ctypes.c_void_p):
        return x.value
    raise TypeError(f"cannot take the address of {type(x)!r}")


def version() -> str:
    return lib().sift_version().decode()


# ----------------------------------------------------- reference interface --

def cublas_2nn_sift(q_points, r_points, type, q_n, r_n, matches, threshold, handle=None, stream_n=1, use=0,
                    warps=17) -> int:
    """Exact 2-NN + ratio test (reference src/knn_brute.cu:24). Returns the status code."""
    return lib().cublas_2nn_sift(_ptr(q_points), _ptr(r_points), type, q_n, r_n, _ptr(matches), threshold,
                                 _ptr(handle), stream_n, use, warps)


def cublas_2nn_f(q_points, r_points, q_n, r_n, sorted, handle=None) -> None:
    """2-NN ranked by -2 q.r into float4 {d1, d2, i1, i2} (reference src/knn_brute.cu:523)."""
    lib().cublas_2nn_f(_ptr(q_points), _ptr(r_points), q_n, r_n, _ptr(sorted), _ptr(handle))
    check(lib().sift_last_status(), "cublas_2nn_f")


def device_brute(q_points, r_points, q_n, r_n, sorted) -> None:
    """Exact squared-L2 2-NN into float4 {d1, d2, i1, i2} (reference src/knn_brute.cu:619)."""
    lib().device_brute(_ptr(q_points), _ptr(r_points), q_n, r_n, _ptr(sorted))
    check(lib().sift_last_status(), "device_brute")


def host_brute(q_points, r_points, q_points_size, r_points_size, sorted) -> None:
    """host_brute contract (reference src/knn_brute.cu:801) computed on the GPU for host arrays."""
    lib().host_brute(_ptr(q_points), _ptr(r_points), q_points_size, r_points_size, _ptr(sorted))
    check(lib().sift_last_status(), "host_brute")


def lsh_gpu(q_points, r_points, type, q_n, r_n, matches, threshold, handle=None, stream_n=2, l=1, lsh_type=0,
            nbits=16) -> int:
    """Random-hyperplane LSH 2-NN (reference src/lsh_h.cu:722). Returns the status code."""
    return lib().lsh_gpu(_ptr(q_points), _ptr(r_points), type, q_n, r_n, _ptr(matches), threshold, _ptr(handle),
                         stream_n, l, lsh_type, nbits)


def stream_status(stream=None) -> int:
    return lib().sift_stream_status(_ptr(stream) if stream is not None else None)


# -------------------------------------------------------- native interface --

def match(q, r, threshold: float = 0.8, metric: int = METRIC_L2, stream=None, outputs=("matches", "nn_idx", "nn_dist")):
    """Exact 2-NN of CUDA tensors q [n, 128] and r [m, 128].

    uint8 rows are searched by the u8 tensor-core kernel; float16 rows by the
    FP16 kernel in place; float32 rows are packed to u8 first. Float values
    must be integers in [0, 255] times one common power of two.
    Returns a dict with the requested outputs as CUDA tensors: ``matches``
    (uint32 -- an int32 tensor viewed as uint32 where torch has that dtype;
    UINT32_MAX where the ratio test fails), ``nn_idx``
    [n, 2] int32 (-1 absent), ``nn_dist`` [n, 2] float32, ``sorted`` [n, 4].
    Asynchronous on ``stream`` (a torch.cuda.Stream or None for the current one)
    for uint8 inputs; float inputs synchronise once to validate the values.
    """
    import torch

    types = {torch.uint8: U8_DEVICE, torch.float16: HALF_DEVICE, torch.float32: FLOAT_DEVICE}
    if q.dtype != r.dtype or q.dtype not in types or not q.is_cuda or not r.is_cuda:
        raise TypeError("match() expects two CUDA tensors of one dtype: uint8, float16 or float32")
    if q.dim() != 2 or q.shape[1] != 128 or r.dim() != 2 or r.shape[1] != 128:
        raise ValueError("descriptors must be [n, 128]")
    q = q.contiguous()
    r = r.contiguous()
    n = q.shape[0]
    dev = q.device
    out = {}
    if "matches" in outputs:
        out["matches"] = torch.empty(n, dtype=torch.int32, device=dev)
    if "nn_idx" in outputs:
        out["nn_idx"] = torch.empty((n, 2), dtype=torch.int32, device=dev)
    if "nn_dist" in outputs:
        out["nn_dist"] = torch.empty((n, 2), dtype=torch.float32, device=dev)
    if "sorted" in outputs:
        out["sorted"] = torch.empty((n, 4), dtype=torch.float32, device=dev)
    s = stream if stream is not None else torch.cuda.current_stream(dev)
    with torch.cuda.device(dev):
        rc = lib().sift2nn_match(q.data_ptr(), r.data_ptr(), types[q.dtype], n, r.shape[0], metric, threshold,
                                 _ptr(out.get("matches")), _ptr(out.get("sorted")), _ptr(out.get("nn_idx")),
                                 _ptr(out.get("nn_dist")), s.cuda_stream)
    check(rc, "sift2nn_match")
    if "matches" in out:
        out["matches"] = out["matches"].view(torch.uint32) if hasattr(torch, "uint32") else out["matches"]
    return out


def lsh_hash(x, planes, stream=None):
    """LSH codes [L, n] (int32 view of uint32) of uint8 CUDA rows x [n, 128] for int8 planes [L, k, 128]."""
    import torch

    L, k = planes.shape[0], planes.shape[1]
    x = x.contiguous()
    planes = planes.contiguous()
    codes = torch.empty((L, x.shape[0]), dtype=torch.int32, device=x.device)
    s = stream if stream is not None else torch.cuda.current_stream(x.device)
    check(lib().sift_lsh_hash(x.data_ptr(), x.shape[0], planes.data_ptr(), L, k, codes.data_ptr(), s.cuda_stream),
          "sift_lsh_hash")
    return codes


def lsh_buckets(codes, k: int, stream=None):
    """Bucket table of LSH codes [L, n] (CUDA int32 / uint32 view) with k bits
    per table: (start [L, 2^B + 1], order [L, n], ocode [L, n]) as CUDA int32
    tensors, B = min(k, 16) -- group b of table t holds the point ids
    order[t, start[t, b]:start[t, b + 1]] (codes ocode[...]), the points whose
    code's top B bits are b."""
    import torch

    codes = codes.contiguous()
    L, n = codes.shape
    top = min(k, 16)
    start = torch.empty((L, (1 << top) + 1), dtype=torch.int32, device=codes.device)
    order = torch.empty((L, n), dtype=torch.int32, device=codes.device)
    ocode = torch.empty((L, n), dtype=torch.int32, device=codes.device)
    s = stream if stream is not None else torch.cuda.current_stream(codes.device)
    check(lib().sift_lsh_buckets(codes.data_ptr(), n, L, k, start.data_ptr(), order.data_ptr(), ocode.data_ptr(),
                                 s.cuda_stream), "sift_lsh_buckets")
    return start, order, ocode


def lsh_match(q, r, planes, threshold: float = 0.0, stream=None, probes: int = 1, candidates: bool = False):
    """LSH 2-NN of CUDA tensors (uint8, float16 or float32; float values that
    are not integers times a power of two take the FP32 hash and scan) with
    int8 hyperplanes planes [L, k, 128].

    Returns {"matches", "nn_idx", "nn_dist"} like match(); only base rows
    sharing a code with the query in some table are candidates. probes > 1
    also searches, per table, the buckets of the query's code with its
    lowest-margin bits flipped (query-directed multi-probe, up to
    2^min(6, k) codes); candidates=True adds "candidates", the base rows
    compared per query.
    """
    import torch

    types = {torch.uint8: U8_DEVICE, torch.float16: HALF_DEVICE, torch.float32: FLOAT_DEVICE}
    if q.dtype != r.dtype or q.dtype not in types or not q.is_cuda or not r.is_cuda:
        raise TypeError("lsh_match() expects two CUDA tensors of one dtype: uint8, float16 or float32")
    L, k = planes.shape[0], planes.shape[1]
    q, r, planes = q.contiguous(), r.contiguous(), planes.contiguous()
    n = q.shape[0]
    out = {"matches": torch.empty(n, dtype=torch.int32, device=q.device),
           "nn_idx": torch.empty((n, 2), dtype=torch.int32, device=q.device),
           "nn_dist": torch.empty((n, 2), dtype=torch.float32, device=q.device)}
    if candidates:
        out["candidates"] = torch.empty(n, dtype=torch.int32, device=q.device)
    s = stream if stream is not None else torch.cuda.current_stream(q.device)
    check(lib().sift_lsh_match_probes(q.data_ptr(), r.data_ptr(), types[q.dtype], n, r.shape[0], planes.data_ptr(), L, k,
                                      probes, threshold, out["matches"].data_ptr(), out["nn_idx"].data_ptr(),
                                      out["nn_dist"].data_ptr(), _ptr(out.get("candidates")), s.cuda_stream),
          "sift_lsh_match_probes")
    return out


# ------------------------------------------------------------------ batches --

def _pairs_array(pairs):
    """(n, 3) uint32 rows {n_q, n_r, r_off} as a contiguous array (sift_pair[])."""
    import numpy as np

    a = np.ascontiguousarray(np.asarray(pairs, dtype=np.uint32).reshape(-1, 3))
    return a


def _batch_outputs(total_q, dev):
    import torch

    return {"matches": torch.empty(total_q, dtype=torch.int32, device=dev),
            "nn_idx": torch.empty((total_q, 2), dtype=torch.int32, device=dev),
            "nn_dist": torch.empty((total_q, 2), dtype=torch.float32, device=dev)}


def match_batch(q, r, pairs, threshold: float = 0.8, stream=None):
    """Exact 2-NN of many problems in one launch.

    q: uint8 CUDA tensor, the query sets of all problems concatenated in
    order; r: uint8 CUDA tensor of base rows; pairs: rows {n_q, n_r, r_off}.
    Returns {"matches", "nn_idx", "nn_dist"} per query row (indices local to
    the problem's base rows).
    """
    import torch

    pa = _pairs_array(pairs)
    total_q = int(pa[:, 0].sum()) if len(pa) else 0
    if q.shape[0] != total_q:
        raise ValueError(f"q has {q.shape[0]} rows, the pairs {total_q}")
    out = _batch_outputs(total_q, q.device)
    s = stream if stream is not None else torch.cuda.current_stream(q.device)
    check(lib().sift2nn_match_batch(_ptr(q), _ptr(r), r.shape[0], pa.ctypes.data, len(pa), threshold,
                                    _ptr(out["matches"]), _ptr(out["nn_idx"]), _ptr(out["nn_dist"]), s.cuda_stream),
          "sift2nn_match_batch")
    return out


def match_mutual_batch(a, b, pairs, threshold: float = 0.8, stream=None):
    """Mutual nearest neighbours of the two sets of many problems (image
    pairs) in two batched searches and one cross-check.

    a: uint8 CUDA tensor, every problem's first set concatenated in order;
    b: uint8 CUDA tensor holding the second sets; pairs: rows {n_a, n_b,
    b_off}. Returns {"matches", "nn_idx", "nn_dist"} per row of a: matches[i]
    = j (local to the problem's set in b) for mutual nearest neighbours that
    pass the forward ratio test when threshold > 0, else 0xFFFFFFFF; nn_idx and
    nn_dist are the forward 2-NN.
    """
    import torch

    pa = _pairs_array(pairs)
    total = int(pa[:, 0].sum()) if len(pa) else 0
    if a.shape[0] != total:
        raise ValueError(f"a has {a.shape[0]} rows, the pairs {total}")
    out = _batch_outputs(total, a.device)
    s = stream if stream is not None else torch.cuda.current_stream(a.device)
    check(lib().sift2nn_match_mutual_batch(_ptr(a), _ptr(b), b.shape[0], pa.ctypes.data, len(pa), threshold,
                                           _ptr(out["matches"]), _ptr(out["nn_idx"]), _ptr(out["nn_dist"]),
                                           s.cuda_stream),
          "sift2nn_match_mutual_batch")
    return out


def compact_matches(out, pairs, capacity=None, stream=None):
    """Per-problem match lists for geometric verification from the outputs
    of match_batch / match_mutual_batch (dict with "matches" and optionally
    "nn_dist"). Returns {"pair", "a", "b" (int64), "d1", "d2" (float32)} over
    all matches, grouped by problem with rows in order, and "offsets"
    ([n_pairs + 1], first match of each problem, then the count)."""
    import torch

    pa = _pairs_array(pairs)
    m = out["matches"]
    rows = m.shape[0]
    cap = rows if capacity is None else int(capacity)
    rec = torch.empty((max(cap, 1), 5), dtype=torch.int32, device=m.device)  # sift_match = 5 x 4 bytes
    offs = torch.empty(len(pa) + 1, dtype=torch.int32, device=m.device)
    s = stream if stream is not None else torch.cuda.current_stream(m.device)
    check(lib().sift_compact_matches(_ptr(m), _ptr(out.get("nn_dist")), rows, pa.ctypes.data, len(pa), _ptr(rec), cap,
                                     _ptr(offs), s.cuda_stream), "sift_compact_matches")
    n = min(int(offs[-1].item()), cap)
    r = rec[:n]
    return {"pair": r[:, 0].long(), "a": r[:, 1].long(), "b": r[:, 2].long(),
            "d1": r[:, 3].view(torch.float32), "d2": r[:, 4].view(torch.float32), "offsets": offs.long()}


def match_mutual(a, b, threshold: float = 0.8, stream=None):
    """Mutual nearest neighbours of one pair of descriptor sets (uint8 CUDA
    tensors [n, 128]); see match_mutual_batch."""
    return match_mutual_batch(a, b, [[a.shape[0], b.shape[0], 0]], threshold, stream)


class BatchPlan:
    """A batch bound to (q, r, outputs) and replayed as one CUDA graph."""

    def __init__(self, q, r, pairs, threshold: float = 0.8, tune: bool = True, shape=None):
        self._pa = _pairs_array(pairs)
        total_q = int(self._pa[:, 0].sum()) if len(self._pa) else 0
        if q.shape[0] != total_q:
            raise ValueError(f"q has {q.shape[0]} rows, the pairs {total_q}")
        self.q, self.r = q, r
        self.out = _batch_outputs(total_q, q.device)
        flags = (SIFT_BATCH_TUNE if tune else 0) | (SIFT_BATCH_SHAPE(shape) if shape is not None else 0)
        h = ctypes.c_void_p()
        check(lib().sift_batch_plan_create(_ptr(q), _ptr(r), r.shape[0], self._pa.ctypes.data, len(self._pa),
                                           threshold, _ptr(self.out["matches"]), _ptr(self.out["nn_idx"]),
                                           _ptr(self.out["nn_dist"]), flags, ctypes.byref(h)), "sift_batch_plan_create")
        self._h = h

    def run(self, stream=None):
        import torch

        s = stream if stream is not None else torch.cuda.current_stream(self.q.device)
        check(lib().sift_batch_plan_run(self._h, s.cuda_stream), "sift_batch_plan_run")
        return self.out

    def info(self):
        qpt, qbuf = ctypes.c_int(), ctypes.c_int()
        ms = (ctypes.c_float * 3)()
        check(lib().sift_batch_plan_info(self._h, ctypes.byref(qpt), ctypes.byref(qbuf), ms), "sift_batch_plan_info")
        return {"qpt": qpt.value, "qbuf": qbuf.value, "tuned_ms": list(ms)}

    def close(self):
        if getattr(self, "_h", None):
            lib().sift_batch_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_describe(pairs, r_rows: int, qpt: int = 2, workers: int = 74):
    """Host-side decomposition of a batch (no GPU): units, records, queries,
    max_splits, grid, group_rows."""
    pa = _pairs_array(pairs)
    out = (ctypes.c_longlong * 6)()
    check(lib().sift_batch_describe(pa.ctypes.data if len(pa) else None, len(pa), r_rows, qpt, workers, out),
          "sift_batch_describe")
    return dict(zip(("units", "tiles", "queries", "max_splits", "grid", "group_rows"), list(out)))


# ------------------------------------------------------------- learned hash --

class MlpHash:
    """A learned hash model (MLP 128 -> 256 -> k, BF16 weights) on the GPU.

    Build it with :meth:`train` (neighbour pairs labelled by the exact search)
    or from explicit FP32 parameters (:meth:`from_params`, the flat layout of
    SIFT_MLP_PARAMS floats).
    """

    def __init__(self, w1, b1, w2, b2, k: int, params=None, loss_curve=None):
        self.w1, self.b1, self.w2, self.b2, self.k = w1, b1, w2, b2, k
        self.params = params
        self.loss_curve = loss_curve
        self._c = sift_mlp(w1.data_ptr(), b1.data_ptr(), w2.data_ptr(), b2.data_ptr(), k)

    @staticmethod
    def _empty(k, dev):
        import torch

        return (torch.empty((256, 128), dtype=torch.bfloat16, device=dev), torch.empty(256, device=dev),
                torch.empty((k, 256), dtype=torch.bfloat16, device=dev), torch.empty(k, device=dev))

    @classmethod
    def train(cls, base, train_q, k: int = 16, steps: int = 1000, batch: int = 2048, lr: float = 2e-3,
              neg_weight: float = 1.0, balance_weight: float = 1.0, seed: int = 0):
        import numpy as np
        import torch

        w1, b1, w2, b2 = cls._empty(k, base.device)
        params = torch.empty(SIFT_MLP_PARAMS, device=base.device)
        curve = np.zeros(max(steps, 1), np.float32)
        check(lib().sift_mlp_train(_ptr(base), base.shape[0], _ptr(train_q), train_q.shape[0], k, steps, batch, lr,
                                   neg_weight, balance_weight, seed, _ptr(w1), _ptr(b1), _ptr(w2), _ptr(b2),
                                   _ptr(params), curve.ctypes.data), "sift_mlp_train")
        return cls(w1, b1, w2, b2, k, params=params, loss_curve=curve[:steps])

    @classmethod
    def from_params(cls, params, k: int):
        """Model from flat FP32 parameters (torch CUDA tensor), weights rounded to BF16."""
        import torch

        p = params.float()
        w1 = p[:256 * 128].view(256, 128).to(torch.bfloat16).contiguous()
        b1 = p[256 * 128:256 * 128 + 256].contiguous()
        o = 256 * 128 + 256
        w2 = p[o:o + 32 * 256].view(32, 256)[:k].to(torch.bfloat16).contiguous()
        b2 = p[o + 32 * 256:o + 32 * 256 + k].contiguous()
        return cls(w1, b1, w2, b2, k, params=params)

    def hash(self, x, with_z: bool = False, stream=None):
        import torch

        codes = torch.empty(x.shape[0], dtype=torch.int32, device=x.device)
        z = torch.empty((x.shape[0], self.k), device=x.device) if with_z else None
        s = stream if stream is not None else torch.cuda.current_stream(x.device)
        check(lib().sift_mlp_hash(_ptr(x), x.shape[0], ctypes.byref(self._c), _ptr(codes), _ptr(z), s.cuda_stream),
              "sift_mlp_hash")
        return (codes, z) if with_z else codes

    def match(self, q, r, n_probes: int = 1, min_candidates: int = 0, max_dist: float = 0.0, threshold: float = 0.0,
              stream=None):
        """{"matches", "nn_idx", "nn_dist", "candidates", "fallback"}: learned-hash 2-NN (see sift_mlp_match)."""
        import torch

        n = q.shape[0]
        out = {"matches": torch.empty(n, dtype=torch.int32, device=q.device),
               "nn_idx": torch.empty((n, 2), dtype=torch.int32, device=q.device),
               "nn_dist": torch.empty((n, 2), dtype=torch.float32, device=q.device),
               "candidates": torch.empty(n, dtype=torch.int32, device=q.device)}
        fb = ctypes.c_uint32(0)
        s = stream if stream is not None else torch.cuda.current_stream(q.device)
        check(lib().sift_mlp_match(_ptr(q), _ptr(r), n, r.shape[0], ctypes.byref(self._c), n_probes, min_candidates,
                                   max_dist, threshold, _ptr(out["matches"]), _ptr(out["nn_idx"]), _ptr(out["nn_dist"]),
                                   _ptr(out["candidates"]), ctypes.byref(fb), s.cuda_stream), "sift_mlp_match")
        out["fallback"] = fb.value
        return out


class HashIndex:
    """A base hashed and bucketed once, searched many times (sift_index_*).

    ``HashIndex.lsh(r, planes)`` uses int8 hyperplanes [L, k, 128];
    ``HashIndex.mlp(r, model)`` a trained :class:`MlpHash`. The index reads
    the base tensor ``r`` (uint8 [n, 128] on the GPU) by reference and keeps
    it alive.
    """

    def __init__(self, handle, r, k: int, L: int, keep=None):
        self._h = handle
        self.r, self.k, self.L = r, k, L
        self._keep = keep

    @classmethod
    def lsh(cls, r, planes):
        r = r.contiguous()
        planes = planes.contiguous()
        h = ctypes.c_void_p()
        check(lib().sift_lsh_index_create(_ptr(r), r.shape[0], _ptr(planes), planes.shape[0], planes.shape[1],
                                          ctypes.byref(h)), "sift_lsh_index_create")
        return cls(h, r, planes.shape[1], planes.shape[0])

    @classmethod
    def mlp(cls, r, model: "MlpHash"):
        r = r.contiguous()
        h = ctypes.c_void_p()
        check(lib().sift_mlp_index_create(_ptr(r), r.shape[0], ctypes.byref(model._c), ctypes.byref(h)),
              "sift_mlp_index_create")
        return cls(h, r, model.k, 1)

    def search(self, q, probes: int = 1, min_candidates: int = 0, max_dist: float = 0.0, threshold: float = 0.0,
               stream=None):
        """{"matches", "nn_idx", "nn_dist", "candidates", "fallback"} for uint8 CUDA queries q [n, 128]."""
        import torch

        q = q.contiguous()
        n = q.shape[0]
        out = {"matches": torch.empty(n, dtype=torch.int32, device=q.device),
               "nn_idx": torch.empty((n, 2), dtype=torch.int32, device=q.device),
               "nn_dist": torch.empty((n, 2), dtype=torch.float32, device=q.device),
               "candidates": torch.empty(n, dtype=torch.int32, device=q.device)}
        fb = ctypes.c_uint32(0)
        s = stream if stream is not None else torch.cuda.current_stream(q.device)
        check(lib().sift_index_search(self._h, _ptr(q), n, probes, min_candidates, max_dist, threshold,
                                      _ptr(out["matches"]), _ptr(out["nn_idx"]), _ptr(out["nn_dist"]),
                                      _ptr(out["candidates"]), ctypes.byref(fb), s.cuda_stream), "sift_index_search")
        out["fallback"] = fb.value
        return out

    def buckets(self, stream=None):
        """The bucket table as CUDA int32 tensors (start [L, 2^B + 1], order [L, n],
        ocode [L, n]) and its group bits B, laid out as :func:`lsh_buckets`."""
        import torch

        top = ctypes.c_int(0)
        check(lib().sift_index_buckets(self._h, None, None, None, ctypes.byref(top), None), "sift_index_buckets")
        dev, n = self.r.device, self.r.shape[0]
        start = torch.empty((self.L, (1 << top.value) + 1), dtype=torch.int32, device=dev)
        order = torch.empty((self.L, n), dtype=torch.int32, device=dev)
        ocode = torch.empty((self.L, n), dtype=torch.int32, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        check(lib().sift_index_buckets(self._h, _ptr(start), _ptr(order), _ptr(ocode), ctypes.byref(top),
                                       s.cuda_stream), "sift_index_buckets")
        return start, order, ocode, top.value

    def close(self):
        if self._h is not None and self._h.value:
            lib().sift_index_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mlp_loss_grad(x, batch: int, k: int, params, neg_weight: float = 1.0, balance_weight: float = 1.0):
    """(loss[4], grads) of one training step on rows x [3 * batch, 128] (device)."""
    import numpy as np
    import torch

    grads = torch.empty(SIFT_MLP_PARAMS, device=x.device)
    loss = (ctypes.c_float * 4)()
    check(lib().sift_mlp_loss_grad(_ptr(x), batch, k, _ptr(params), neg_weight, balance_weight, _ptr(grads), loss),
          "sift_mlp_loss_grad")
    return np.array(list(loss), np.float64), grads
