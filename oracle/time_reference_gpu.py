"""Times the reference's own GPU exact functions (checker-side measurement, not
the product): cublas_2nn_sift (type FLOAT_DEVICE, inputs / 512 and the batch
settings of src/test.cu:103,210), cublas_2nn_f and device_brute, built from the
reference sources into oracle/_ref/libref.so, on the 10,000 x 1,000,000
generator workload, with CUDA events around each synchronous call.

  python oracle/time_reference_gpu.py [--out FILE]

device_brute runs a 200-query sample (its one batch of 800 MB distances) and
is scaled to 10,000 queries.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from matching_sift_b200 import datagen  # noqa: E402


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--out")
    args = ap.parse_args()
    dev = torch.device("cuda:0")
    ref = oracle.ref()
    base = datagen.make_base(1_000_000, seed=0)
    q = datagen.make_queries(10_000, base, seed=0)
    q_n, r_n = q.shape[0], base.shape[0]

    def timed(fn, reps):
        ts = []
        for _ in range(reps):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            rc = fn()
            b.record()
            torch.cuda.synchronize()
            assert rc == 0, rc
            ts.append(a.elapsed_time(b))
        return ts

    out = {}
    qs = torch.from_numpy(q.astype(np.float32) / 512.0).to(dev)
    rs = torch.from_numpy(base.astype(np.float32) / 512.0).to(dev)
    m = torch.zeros(q_n, dtype=torch.int32, device=dev)
    t = timed(lambda: ref.ref_cublas_2nn_sift(qs.data_ptr(), rs.data_ptr(), q_n, r_n, m.data_ptr(), 0.8, 1,
                                              2 * r_n * 383, 17), 3)
    out["cublas_2nn_sift_ms"] = t
    del qs, rs
    qf = torch.from_numpy(q.astype(np.float32)).to(dev)
    rf = torch.from_numpy(base.astype(np.float32)).to(dev)
    s = torch.zeros((q_n, 4), dtype=torch.float32, device=dev)
    out["cublas_2nn_f_ms"] = timed(lambda: ref.ref_cublas_2nn_f(qf.data_ptr(), rf.data_ptr(), q_n, r_n, s.data_ptr()),
                                   2)
    s2 = torch.zeros((200, 4), dtype=torch.float32, device=dev)
    t = timed(lambda: ref.ref_device_brute(qf.data_ptr(), rf.data_ptr(), 200, r_n, s2.data_ptr()), 1)
    out["device_brute_200q_ms"] = t
    out["device_brute_10000q_ms_scaled"] = [x * q_n / 200 for x in t]
    out["queries_per_s"] = {"cublas_2nn_sift": q_n / (min(out["cublas_2nn_sift_ms"]) * 1e-3),
                            "cublas_2nn_f": q_n / (min(out["cublas_2nn_f_ms"]) * 1e-3),
                            "device_brute": 200 / (min(t) * 1e-3)}
    line = json.dumps(out)
    print(line)
    if args.out:
        with open(args.out, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
