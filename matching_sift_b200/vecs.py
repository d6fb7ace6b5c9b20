"""Descriptor files in the TEXMEX formats (ANN_SIFT1M / ANN_SIFT1B).

The reference benchmark reads ``sift_base.fvecs`` / ``sift_query.fvecs`` and
``sift_groundtruth.ivecs`` record by record (src/test.cu:76-155): every record
is a little-endian int32 dimension followed by that many float32 (``.fvecs``),
uint8 (``.bvecs``) or int32 (``.ivecs``) values. The reference checks each
dimension against 128 and, for its float path, divides the values by 512
(src/test.cu:96-103); the ground truth keeps the first `recall` of the 100 ids
per query (src/test.cu:136-146). Its recall tally (src/test.cu:221-296)
counts, per query, whether the match is missing from the first 1, 10, 20, ...,
100 true neighbours.

Here the files are memory-mapped and decoded in one pass. SIFT descriptors
are integers in [0, 255] stored as floats, so ``to_u8`` turns them into the
u8 rows the search kernels take, exactly and only when every value is such an
integer.
"""
from __future__ import annotations

import os

import numpy as np

_DTYPES = {".fvecs": np.dtype("<f4"), ".bvecs": np.dtype("u1"), ".ivecs": np.dtype("<i4")}


def _kind(path, kind):
    if kind is None:
        kind = os.path.splitext(str(path))[1].lower()
    if kind not in _DTYPES:
        raise ValueError(f"unknown vector file kind {kind!r} (expected .fvecs, .bvecs or .ivecs)")
    return kind


def read_vecs(path, count: int | None = None, start: int = 0, dim: int | None = None, kind: str | None = None):
    """Records [start, start + count) of a vecs file as an [n, dim] array.

    The dimension comes from the first record (or must equal `dim`); every
    record read must carry the same dimension, else ValueError (the reference
    prints a warning and reads on).
    """
    kind = _kind(path, kind)
    vt = _DTYPES[kind]
    size = os.path.getsize(path)
    if size < 4:
        if count:
            raise ValueError(f"{path}: empty file")
        return np.zeros((0, dim or 0), dtype=vt)
    with open(path, "rb") as f:
        d0 = int(np.frombuffer(f.read(4), dtype="<i4")[0])
    if d0 <= 0:
        raise ValueError(f"{path}: bad dimension {d0} in the first record")
    if dim is not None and d0 != dim:
        raise ValueError(f"{path}: dimension {d0}, expected {dim}")
    rec = np.dtype([("d", "<i4"), ("v", vt, (d0,))])
    n_total = size // rec.itemsize
    if size % rec.itemsize:
        raise ValueError(f"{path}: size {size} is not a multiple of the record size {rec.itemsize}")
    if start < 0 or start > n_total:
        raise ValueError(f"{path}: start {start} outside [0, {n_total}]")
    n = n_total - start if count is None else count
    if n < 0 or start + n > n_total:
        raise ValueError(f"{path}: {n} records from {start} requested, the file holds {n_total}")
    mm = np.memmap(path, dtype=rec, mode="r", offset=start * rec.itemsize, shape=(n,))
    if n and not np.all(mm["d"] == d0):
        bad = int(np.flatnonzero(mm["d"] != d0)[0])
        raise ValueError(f"{path}: record {start + bad} has dimension {int(mm['d'][bad])}, expected {d0}")
    return np.array(mm["v"], copy=True)


def read_fvecs(path, count=None, start=0, dim=None):
    return read_vecs(path, count, start, dim, ".fvecs")


def read_bvecs(path, count=None, start=0, dim=None):
    return read_vecs(path, count, start, dim, ".bvecs")


def read_ivecs(path, count=None, start=0, k=None):
    """Ground truth: the first `k` ids of each record (all when k is None)."""
    x = read_vecs(path, count, start, None, ".ivecs")
    if k is not None:
        if k > x.shape[1]:
            raise ValueError(f"{path}: {x.shape[1]} ids per record, {k} requested")
        x = x[:, :k]
    return x


def write_vecs(path, x, kind: str | None = None):
    """Writes rows of x as records of `kind` (from the extension by default)."""
    kind = _kind(path, kind)
    vt = _DTYPES[kind]
    x = np.asarray(x)
    if x.ndim != 2:
        raise ValueError("write_vecs takes an [n, dim] array")
    rec = np.zeros(x.shape[0], dtype=[("d", "<i4"), ("v", vt, (x.shape[1],))])
    rec["d"] = x.shape[1]
    rec["v"] = x
    rec.tofile(path)


def to_u8(x):
    """[n, d] descriptors with integer values in [0, 255] (as SIFT stores them
    in .fvecs) -> uint8, exactly; ValueError when a value is not such an
    integer."""
    x = np.asarray(x)
    if x.dtype == np.uint8:
        return x
    if x.size and (not np.all(np.isfinite(x)) or x.min() < 0 or x.max() > 255 or np.any(x != np.round(x))):
        raise ValueError("values are not integers in [0, 255]; the u8 search cannot represent them exactly")
    return x.astype(np.uint8)


def scaled_half(x, scale: float = 1.0 / 512):
    """The reference's FP16 input convention: values times `scale` (1/512 in
    src/test.cu:100) stored as float16."""
    return (np.asarray(x, dtype=np.float32) * np.float32(scale)).astype(np.float16)


RECALL_RANKS = (1, 10, 20, 30, 40, 50, 60, 70, 80, 90, 100)


def recall_misses(matches, truth, ranks=RECALL_RANKS):
    """For each rank r: the number of queries whose match is not among their
    first r true neighbours (truth: [q, >= max(ranks)] ids; matches: [q]
    ids, a no-match value counting as a miss everywhere)."""
    m = np.asarray(matches).astype(np.int64).reshape(-1)
    t = np.asarray(truth).astype(np.int64)
    if t.shape[0] != m.shape[0]:
        raise ValueError(f"{m.shape[0]} matches, {t.shape[0]} ground-truth rows")
    if max(ranks) > t.shape[1]:
        raise ValueError(f"ground truth has {t.shape[1]} ids per query, rank {max(ranks)} requested")
    hit = t == m[:, None]
    first = np.where(hit.any(1), hit.argmax(1), t.shape[1])  # rank position of the match, or past the end
    return {r: int(np.count_nonzero(first >= r)) for r in ranks}


def recall_at(matches, truth, r: int = 1) -> float:
    """Fraction of queries whose match is among their first r true neighbours."""
    n = np.asarray(matches).reshape(-1).shape[0]
    return 1.0 - recall_misses(matches, truth, (r,))[r] / max(n, 1)
