"""Seeded synthetic SIFT-like descriptors (stand-in for ANN_SIFT1M, which is absent).

The reference benchmark reads ANN_SIFT1M ``.fvecs`` files (src/test.cu:76-155);
those files are not available here, so every workload is generated from a seed
with the following published recipe:

* base vector: 128 draws of Exponential(1); exactly 38 (= round(0.3 * 128))
  positions chosen uniformly at random are set to zero; the vector is scaled to
  L2 norm 512, rounded half-to-even and clamped to [0, 255]; stored as uint8.
* query set: half of the queries (positions chosen by a random permutation) are
  copies of uniformly chosen base rows plus N(0, 8^2) noise, rounded and
  clamped; the other half are fresh draws of the base recipe.

Random streams: numpy PCG64 (``np.random.default_rng``) seeded with
``[seed, stream]`` where stream 0 draws the base, 1 the queries, so the same
seed reproduces the same bytes on every machine with numpy >= 1.17.
"""
from __future__ import annotations

import numpy as np

DIM = 128
ZEROED = 38          # round(0.3 * 128)
TARGET_NORM = 512.0
NOISE_SIGMA = 8.0
_CHUNK = 1 << 16


def _fresh(rng: np.random.Generator, n: int) -> np.ndarray:
    out = np.empty((n, DIM), np.uint8)
    for s in range(0, n, _CHUNK):
        m = min(_CHUNK, n - s)
        x = rng.standard_exponential((m, DIM))
        drop = np.argpartition(rng.random((m, DIM)), ZEROED, axis=1)[:, :ZEROED]
        np.put_along_axis(x, drop, 0.0, axis=1)
        nrm = np.linalg.norm(x, axis=1, keepdims=True)
        nrm[nrm == 0] = 1.0
        out[s:s + m] = np.clip(np.rint(x * (TARGET_NORM / nrm)), 0, 255).astype(np.uint8)
    return out


def make_base(n: int, seed: int = 0) -> np.ndarray:
    """n x 128 uint8 base descriptors."""
    return _fresh(np.random.default_rng([seed, 0]), n)


def make_queries(n: int, base: np.ndarray, seed: int = 0, copy_frac: float = 0.5,
                 sigma: float = NOISE_SIGMA) -> np.ndarray:
    """n x 128 uint8 queries: ``copy_frac`` noisy copies of base rows, the rest fresh."""
    rng = np.random.default_rng([seed, 1])
    n_copy = int(round(n * copy_frac))
    perm = rng.permutation(n)
    out = np.empty((n, DIM), np.uint8)
    if n_copy:
        src = rng.integers(0, base.shape[0], n_copy)
        noisy = base[src].astype(np.float64) + rng.normal(0.0, sigma, (n_copy, DIM))
        out[perm[:n_copy]] = np.clip(np.rint(noisy), 0, 255).astype(np.uint8)
    if n - n_copy:
        out[perm[n_copy:]] = _fresh(rng, n - n_copy)
    return out


def query_copies(n: int, seed: int = 0, copy_frac: float = 0.5) -> np.ndarray:
    """Boolean mask of the queries of ``make_queries(n, ..., seed, copy_frac)``
    that are noisy copies of base rows (the rest are fresh draws)."""
    rng = np.random.default_rng([seed, 1])
    n_copy = int(round(n * copy_frac))
    perm = rng.permutation(n)
    mask = np.zeros(n, bool)
    mask[perm[:n_copy]] = True
    return mask


def make_workload(n_query: int, n_base: int, seed: int = 0):
    """(queries, base) as uint8 arrays from the recipe above."""
    base = make_base(n_base, seed)
    return make_queries(n_query, base, seed), base


def make_hyperplanes(nbits: int, n_tables: int = 1, seed: int = 0) -> np.ndarray:
    """[n_tables, nbits, 128] float32 N(0, 1) hyperplanes from a fixed seed."""
    rng = np.random.default_rng([seed, 2])
    return rng.standard_normal((n_tables, nbits, DIM)).astype(np.float32)


def quantize_planes(planes: np.ndarray, scale: float = 32.0) -> np.ndarray:
    """int8 hyperplanes: rint(planes * scale) clamped to [-127, 127].

    The LSH kernels compute exact integer dot products (u8 x s8 on the tensor
    cores), so hyperplanes are used in this quantised form everywhere.
    """
    return np.clip(np.rint(planes * scale), -127, 127).astype(np.int8)


def make_pairs(n_pairs: int, lo: int = 500, hi: int = 8000, seed: int = 0, overlap: float = 0.4):
    """Image pairs with uneven keypoint counts (log-uniform in [lo, hi]).

    In every pair ``overlap`` of side B's descriptors are noisy copies (sigma 8)
    of side A's. Returns a list of (a, b) uint8 arrays.
    """
    rng = np.random.default_rng([seed, 3])
    pairs = []
    for _ in range(n_pairs):
        na, nb = np.exp(rng.uniform(np.log(lo), np.log(hi), 2)).astype(np.int64)
        a = _fresh(rng, int(na))
        b = _fresh(rng, int(nb))
        k = int(round(overlap * nb))
        if k:
            pos = rng.choice(int(nb), k, replace=False)
            src = rng.integers(0, int(na), k)
            noisy = a[src].astype(np.float64) + rng.normal(0.0, NOISE_SIGMA, (k, DIM))
            b[pos] = np.clip(np.rint(noisy), 0, 255).astype(np.uint8)
        pairs.append((a, b))
    return pairs
