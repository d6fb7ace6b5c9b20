"""Generate the golden fixtures of tests/golden from the reference implementation.

The reference publishes no golden vectors, so fixtures are produced by running
the reference's own functions (compiled unmodified from its sources into
oracle/_ref/libref.so by ``make -C oracle ref``) on seeded inputs:

  python tests/golden/make_golden.py          # CPU: host_brute (src/knn_brute.cu:801)
  python tests/golden/make_golden.py --gpu    # GPU: device_brute, cublas_2nn_f, cublas_2nn_sift

Each fixture is a compressed .npz holding the inputs (uint8) and the
reference's raw outputs.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from matching_sift_b200 import datagen  # noqa: E402


def cpu_cases():
    """(name, q, r) u8 inputs covering the generator and the tie / size edges."""
    cases = []
    q, r = datagen.make_workload(96, 2048, seed=11)
    cases.append(("gen_96x2048", q, r))
    # duplicated base rows and queries that equal base rows: distance ties
    rng = np.random.default_rng(5)
    base = datagen.make_base(64, seed=12)
    r = np.concatenate([base, base[::-1], base[:16]], axis=0)          # every row appears 2-3 times
    q = np.concatenate([base[:8], r[[3, 70, 129]], datagen.make_base(8, seed=13)], axis=0)
    cases.append(("ties_19x144", q, r))
    # extreme values: all-0 / all-255 rows, the largest possible distance
    r = np.stack([np.zeros(128, np.uint8), np.full(128, 255, np.uint8), np.full(128, 1, np.uint8)])
    q = np.stack([np.full(128, 255, np.uint8), np.zeros(128, np.uint8), rng.integers(0, 256, 128, dtype=np.uint8)])
    cases.append(("extremes_3x3", q, r))
    # single base row (no second neighbour) and two base rows
    q, r = datagen.make_workload(5, 1, seed=14)
    cases.append(("one_base_5x1", q, r))
    q, r = datagen.make_workload(3, 2, seed=15)
    cases.append(("two_base_3x2", q, r))
    # ragged sizes around the tile edges (128 queries, 256 base rows)
    q, r = datagen.make_workload(129, 257, seed=16)
    cases.append(("ragged_129x257", q, r))
    return cases


def make_cpu():
    for name, q, r in cpu_cases():
        out = oracle.ref_host_brute(q.astype(np.float32), r.astype(np.float32), nthreads=4)
        path = os.path.join(HERE, f"host_brute_{name}.npz")
        np.savez_compressed(path, q=q, r=r, sorted=out)
        print("wrote", path, q.shape, r.shape)


def make_gpu(out_dir: str):
    import torch

    ref = oracle.ref()
    dev = torch.device("cuda:0")
    os.makedirs(out_dir, exist_ok=True)
    for name, q, r in cpu_cases()[:1] + [("gen_200x5000", *datagen.make_workload(200, 5000, seed=21))]:
        qf = torch.from_numpy(q.astype(np.float32)).to(dev)
        rf = torch.from_numpy(r.astype(np.float32)).to(dev)
        res = {"q": q, "r": r}
        s = torch.empty((q.shape[0], 4), dtype=torch.float32, device=dev)
        assert ref.ref_device_brute(qf.data_ptr(), rf.data_ptr(), q.shape[0], r.shape[0], s.data_ptr()) == 0
        res["device_brute"] = s.cpu().numpy()
        s = torch.empty((q.shape[0], 4), dtype=torch.float32, device=dev)
        assert ref.ref_cublas_2nn_f(qf.data_ptr(), rf.data_ptr(), q.shape[0], r.shape[0], s.data_ptr()) == 0
        res["cublas_2nn_f"] = s.cpu().numpy()
        # cublas_2nn_sift needs the 1/512 scaling of the reference test (src/test.cu:103, :129)
        qs = (qf / 512.0).contiguous()
        rs = (rf / 512.0).contiguous()
        m = torch.empty(q.shape[0], dtype=torch.int32, device=dev)
        rows = q.shape[0]
        assert ref.ref_cublas_2nn_sift(qs.data_ptr(), rs.data_ptr(), rows, r.shape[0], m.data_ptr(), 2.0, 1,
                                       2 * ((r.shape[0] + 15) // 16 * 16) * 383, 17) == 0
        res["cublas_2nn_sift_thr2"] = m.cpu().numpy().view(np.uint32)
        assert ref.ref_cublas_2nn_sift(qs.data_ptr(), rs.data_ptr(), rows, r.shape[0], m.data_ptr(), 0.8, 1,
                                       2 * ((r.shape[0] + 15) // 16 * 16) * 383, 17) == 0
        res["cublas_2nn_sift_thr08"] = m.cpu().numpy().view(np.uint32)
        path = os.path.join(out_dir, f"gpu_ref_{name}.npz")
        np.savez_compressed(path, **res)
        print("wrote", path)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if a.gpu:
        make_gpu(a.out)
    else:
        make_cpu()
