"""Small repeatable workloads of single kernels, for profilers.

    python -m matching_sift_b200.kernel_cases CASE [--reps N]

Each case builds seeded inputs, runs its call once to warm up and N more
times, synchronises and exits 0. Cases and the kernel they exercise:

  fp16       exact2nn_f16_pair_kernel       2,560 x 1,000,000 FP16 rows
  pairs      exact2nn_u8_pair_batch_kernel  128 uneven image pairs, one batch plan
  lsh_hash   lsh_hash_kernel                1,000,000 rows, 8 tables x 16 bits
  lsh_scan   lsh_scan_kernel                2,560 queries, 1,000,000 rows, 4 x 16 bits
  lsh_probe  lsh_scan_kernel                2,560 queries, 1,000,000 rows, 8 x 16 bits, 8 probes
                                            per table (persistent index: the scan without the base hash)
  mlp_hash   mlp_hash_kernel                1,000,000 rows, MLP 128 -> 256 -> 16
  float      exact2nn_float_pair_kernel     2,560 x 1,000,000 general float32 rows (split FP16)
"""
from __future__ import annotations

import argparse

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=("fp16", "pairs", "lsh_hash", "lsh_scan", "lsh_probe", "mlp_hash", "float"))
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()

    import torch

    import matching_sift_b200 as ms
    from matching_sift_b200 import datagen

    dev = torch.device("cuda", 0)
    if args.case == "fp16":
        q, r = datagen.make_workload(2560, 1_000_000, seed=0)
        qd = torch.from_numpy(q).to(dev).half()
        rd = torch.from_numpy(r).to(dev).half()
        run = lambda: ms.match(qd, rd, outputs=("nn_idx",))
    elif args.case == "pairs":
        data = datagen.make_pairs(128, seed=0)
        q = torch.from_numpy(np.concatenate([a for a, _ in data])).to(dev)
        r = torch.from_numpy(np.concatenate([b for _, b in data])).to(dev)
        pairs, off = [], 0
        for a, b in data:
            pairs.append([a.shape[0], b.shape[0], off])
            off += b.shape[0]
        plan = ms.BatchPlan(q, r, pairs, tune=False, shape=0)
        run = plan.run
    elif args.case in ("lsh_hash", "lsh_scan"):
        L = 8 if args.case == "lsh_hash" else 4
        q, r = datagen.make_workload(2560, 1_000_000, seed=0)
        qd, rd = torch.from_numpy(q).to(dev), torch.from_numpy(r).to(dev)
        planes = torch.from_numpy(datagen.quantize_planes(datagen.make_hyperplanes(16, L, seed=1))).to(dev)
        run = (lambda: ms.lsh_hash(rd, planes)) if args.case == "lsh_hash" else (lambda: ms.lsh_match(qd, rd, planes))
    elif args.case == "lsh_probe":
        q, r = datagen.make_workload(2560, 1_000_000, seed=0)
        qd, rd = torch.from_numpy(q).to(dev), torch.from_numpy(r).to(dev)
        planes = torch.from_numpy(datagen.quantize_planes(datagen.make_hyperplanes(16, 8, seed=1))).to(dev)
        index = ms.HashIndex.lsh(rd, planes)
        run = lambda: index.search(qd, probes=8)
    elif args.case == "float":
        g = torch.Generator(device=dev)
        g.manual_seed(3)
        rf = torch.rand((1_000_000, 128), device=dev, generator=g)
        rf /= rf.norm(dim=1, keepdim=True)
        qf = torch.rand((2560, 128), device=dev, generator=g)
        qf /= qf.norm(dim=1, keepdim=True)
        run = lambda: ms.match(qf, rf, outputs=("nn_idx",))
    else:
        # random parameters in the flat SIFT_MLP_PARAMS layout: W1, b1, W2 (32 rows), b2 (32)
        g = np.random.default_rng(1)
        w2 = np.zeros((32, 256))
        w2[:16] = g.normal(0, 0.0884, (16, 256))
        p = np.concatenate([g.normal(0, 0.125, 256 * 128), g.normal(0, 0.3, 256), w2.ravel(),
                            np.concatenate([g.normal(0, 0.1, 16), np.zeros(16)])]).astype(np.float32)
        r = torch.from_numpy(datagen.make_base(1_000_000, seed=0)).to(dev)
        model = ms.MlpHash.from_params(torch.from_numpy(p).to(dev), 16)
        run = lambda: model.hash(r)
    run()
    torch.cuda.synchronize()
    for _ in range(args.reps):
        run()
    torch.cuda.synchronize()
    if ms.stream_status() != ms.SIFT_OK:
        raise SystemExit("device status not OK")


if __name__ == "__main__":
    main()
