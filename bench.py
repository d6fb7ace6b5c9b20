#!/usr/bin/env python
"""Benchmark of the exact 2-NN matching path (one JSON line on rank 0).

Workload: 10,000 queries against a 1,000,000 x 128 uint8 base from the seeded
generator (matching_sift_b200.datagen; stand-in for ANN_SIFT1M), exact
2-NN with the Lowe ratio test at 0.8.

  value : queries/s with inputs resident in HBM, one step = one full
          sift2nn_match call (row norms, fused tensor-core search, merge)
  e2e   : queries/s through the reference-named C ABI call cublas_2nn_sift
          with host uint8 buffers in and a host match array out; the copies
          are inside the timed region
  roofline : the fused search kernel, timed with CUDA events on its own
          stream; 2 * Q * N * 128 integer ops per launch
  cpu_baseline : the reference's own host_brute (compiled from its sources)
          on all host cores over a bounded query sample

Multi-GPU: the path shards by queries with the base replicated, so every rank
matches its own 10,000 queries (weak scaling, no data-path collective).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

Q_N, R_N, DIM = 10_000, 1_000_000, 128
THRESHOLD = 0.8
METRIC = "2-NN queries/s on a 1M×128 base: exact u8 vs FP16 vs learned hash at recall@1≥0.8"
WORKLOAD = "exact 2-NN, 10,000 x 128 u8 queries vs 1,000,000 x 128 u8 base, ratio test 0.8"
L2_BYTES = 126 * 1024 * 1024


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every 5 ms from a thread (read-only queries), else
    nvidia-smi every 200 ms. The timed regions last tens of milliseconds, so
    the 200 ms tool alone sees one sample at most."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index: int, period_s: float = 0.005):
        self.gpu = gpu_index
        self.period = period_s
        self.rows = []  # (sm_mhz, max_mhz, set of reason names)
        self.proc = None
        self._t = None
        self._stop = threading.Event()
        self.source = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:
            import torch
            u = str(torch.cuda.get_device_properties(self.gpu).uuid)
            return pynvml.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(self.gpu)

    def _poll_nvml(self, nv, h):
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        while not self._stop.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((sm, mx, {n for n, b in bits.items() if r & b}))
            except Exception:
                pass
            self._stop.wait(self.period)

    def __enter__(self):
        try:
            import pynvml
            h = self._nvml_handle()
            self._t = threading.Thread(target=self._poll_nvml, args=(pynvml, h), daemon=True)
            self._t.start()
            self.source = "nvml"
            return self
        except Exception:
            self._t = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read_smi, daemon=True)
            self._t.start()
            self.source = "nvidia-smi"
        except OSError:
            self.proc = None
        return self

    def _read_smi(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                mx = float(parts[2]) if parts[2].replace(".", "").isdigit() else float("nan")
                self.rows.append((float(parts[1]), mx,
                                  {self.NAMES[k] for k in range(4) if parts[5 + k].lower() == "active"}))

    def __exit__(self, *exc):
        self._stop.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self._t is not None:
            self._t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [r[0] for r in self.rows]
        mx = [r[1] for r in self.rows if r[1] == r[1]]
        reasons = sorted(set().union(*(r[2] for r in self.rows)))
        return {"sm_mhz": float(np.median(sm)), "sm_min_mhz": min(sm), "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows), "source": self.source}


def _profile_value(name, key):
    """A `key: value` line of a committed profile summary under profiles/, if present."""
    try:
        for line in open(os.path.join(ROOT, "profiles", name)):
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


# ------------------------------------------------------------ CPU baselines --

def _host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_reference_rate(q, r, target_s: float):
    """(queries/s, sample description, threads, kind) of the reference host_brute on a bounded sample."""
    import oracle

    threads = _host_threads()
    rf = np.ascontiguousarray(r, dtype=np.float32)
    kind = "reference"
    if oracle.ref_available():
        def run(n):
            return oracle.ref_host_brute(q[:n].astype(np.float32), rf, nthreads=threads)
    else:
        kind = "port"

        def run(n):
            return oracle.brute_2nn_u8(q[:n], r, nthreads=threads)
    n = threads
    t0 = time.perf_counter()
    run(n)
    dt = time.perf_counter() - t0
    per_q = dt / n
    n2 = int(max(threads, min(q.shape[0], target_s / max(per_q, 1e-9))))
    n2 = max(threads, (n2 // threads) * threads)
    t0 = time.perf_counter()
    run(n2)
    dt = time.perf_counter() - t0
    return n2 / dt, f"{n2} queries x {r.shape[0]} base rows ({dt:.1f} s)", threads, kind


# ----------------------------------------------------------------- main ----

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true", help="time only the device-resident path")
    ap.add_argument("--queries", type=int, default=Q_N, help="queries per GPU (profiling of smaller cases)")
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the FP16, batched-pairs, learned-hash and LSH legs")
    ap.add_argument("--base-file", help="base descriptors (.fvecs/.bvecs, e.g. ANN_SIFT1M sift_base.fvecs; "
                                        "the first 1,000,000 rows) instead of the seeded generator")
    ap.add_argument("--query-file", help="query descriptors (.fvecs/.bvecs; the first --queries rows)")
    ap.add_argument("--truth-file", help="ground truth (.ivecs) for recall of the exact matches")
    args = ap.parse_args()
    if bool(args.base_file) != bool(args.query_file):
        ap.error("--base-file and --query-file go together")
    args.warmup = max(args.warmup, 3)

    world = _env_int("WORLD_SIZE", 1)
    rank = _env_int("RANK", 0)
    local_rank = _env_int("LOCAL_RANK", 0)

    if args.impl == "reference":
        return reference_arm(args, world, rank)

    import torch
    import torch.distributed as dist

    import matching_sift_b200 as ms

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))

    from matching_sift_b200 import datagen

    q_n = args.queries
    if args.base_file:
        from matching_sift_b200 import vecs

        base = vecs.to_u8(vecs.read_vecs(args.base_file, count=R_N, dim=DIM))
        queries = vecs.to_u8(vecs.read_vecs(args.query_file, count=q_n, dim=DIM))
        data_note = (f"descriptor files {os.path.basename(args.base_file)} (first {R_N:,} rows) and "
                     f"{os.path.basename(args.query_file)} (first {q_n:,} rows; the same queries on every rank)")
    else:
        base = datagen.make_base(R_N, seed=0)
        queries = datagen.make_queries(q_n, base, seed=rank)
        data_note = "synthetic (seeded generator standing in for ANN_SIFT1M; base seed 0, queries seed = rank)"
    lib = ms.lib()

    qd = torch.from_numpy(queries).to(dev)
    rd = torch.from_numpy(base).to(dev)
    matches = torch.empty(q_n, dtype=torch.int32, device=dev)
    nn_idx = torch.empty((q_n, 2), dtype=torch.int32, device=dev)
    nn_dist = torch.empty((q_n, 2), dtype=torch.float32, device=dev)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        rc = lib.sift2nn_match(qd.data_ptr(), rd.data_ptr(), ms.U8_DEVICE, q_n, R_N, ms.METRIC_L2, THRESHOLD,
                               matches.data_ptr(), None, nn_idx.data_ptr(), nn_dist.data_ptr(), stream.cuda_stream)
        if rc != 0:
            raise ms.SiftError(rc, "sift2nn_match")

    # ---- device-resident throughput
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if ms.stream_status(stream.cuda_stream) != 0:
        raise RuntimeError("device status after warm-up")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.sift_launch_count()
    lib.sift_profile_enable(1)
    with ClockSampler(local_rank) as clocks:
        for k in range(args.steps):
            flush.fill_(k)  # evict the base from L2 between steps (outside the timed events)
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    lib.sift_profile_enable(0)
    launches = lib.sift_launch_count() - launches0
    import ctypes
    kt, kn = ctypes.c_double(0.0), ctypes.c_int(0)
    lib.sift_profile_collect(ctypes.byref(kt), ctypes.byref(kn))
    if ms.stream_status(stream.cuda_stream) != 0:
        raise RuntimeError("device status after timed steps")
    step_ms = float(sum(a.elapsed_time(b) for a, b in ev))
    kernel_ms = kt.value / max(kn.value, 1)

    # ---- the same search on FP16 rows (kind::f16 kernel), device-resident
    variants = {}
    if not args.no_variants:
        variants["fp16"] = fp16_leg(args, lib, ms, torch, qd, rd, flush, stream, q_n)
        if not torch.equal(variants["fp16"].pop("nn_idx"), nn_idx):
            raise RuntimeError("FP16 and u8 kernels disagree")
        variants["pairs"] = pairs_leg(args, ms, torch, dev, stream)
        variants["mutual"] = mutual_leg(args, ms, torch, dev, stream)
        truth = nn_idx[:, 0].cpu().numpy()
        copies = datagen.query_copies(q_n, seed=rank)
        hbm = _peaks()[0]["hbm_gbs"]
        variants["lsh"] = lsh_leg(args, ms, torch, dev, stream, qd, rd, truth, copies, hbm)
        variants["learned"] = learned_leg(args, ms, torch, dev, stream, qd, rd, base, truth, copies, hbm,
                                          variants["lsh"]["grid"])
        variants["cfg1"] = cfg1_leg(args, ms, torch, dev, stream)
        variants["float"] = float_leg(args, ms, torch, dev, stream, q_n, _peaks()[0]["bf16_tflops"])

    # ---- end to end through the C ABI with host buffers
    e2e_ms = float("nan")
    h2d_ms = float("nan")
    if not args.skip_e2e:
        qh = torch.from_numpy(queries).pin_memory()
        rh = torch.from_numpy(base).pin_memory()
        mh = torch.empty(q_n, dtype=torch.int32).pin_memory()

        def e2e_step():
            rc = lib.cublas_2nn_sift(qh.data_ptr(), rh.data_ptr(), ms.U8_HOST, q_n, R_N, mh.data_ptr(), THRESHOLD,
                                     None, 1, 0, 17)
            if rc != 0:
                raise ms.SiftError(rc, "cublas_2nn_sift")

        for _ in range(args.warmup):
            e2e_step()
        e2e_ms = 0.0
        legacy = torch.cuda.default_stream(dev)
        for k in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(legacy)
            e2e_step()
            b.record(legacy)
            b.synchronize()
            e2e_ms += a.elapsed_time(b)
        np.testing.assert_array_equal(mh.numpy(), matches.cpu().numpy())
        # The PCIe bound of this leg on this box: the same bytes copied from
        # pinned host memory alone (one copy each of queries and base).
        qd2, rd2 = torch.empty_like(qd), torch.empty_like(rd)
        h2d = []
        for _ in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(legacy)
            qd2.copy_(qh, non_blocking=True)
            rd2.copy_(rh, non_blocking=True)
            b.record(legacy)
            b.synchronize()
            h2d.append(a.elapsed_time(b))
        h2d_ms = min(h2d)
        del qd2, rd2

    # ---- max over ranks
    vkeys = sorted(variants)
    t = torch.tensor([step_ms, e2e_ms, kernel_ms] +
                     [variants[k].get(f, 0.0) for k in vkeys for f in ("step_ms", "kernel_ms")],
                     dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    vals = t.tolist()
    step_ms, e2e_ms, kernel_ms = vals[:3]
    for n, k in enumerate(vkeys):
        variants[k]["step_ms"], variants[k]["kernel_ms"] = vals[3 + 2 * n], vals[4 + 2 * n]

    if rank == 0:
        peaks, peak_src = _peaks()
        ops = 2.0 * q_n * R_N * DIM
        achieved = ops / (kernel_ms * 1e-3) / 1e12
        # Dense int8 peak measured on this pool's B200 by matching_sift_b200/peak_int8
        # (profiles/tcgen05_int8_peak.md); MEASURED_PEAKS.json has no int8 figure.
        peak_int8 = _profile_value("tcgen05_int8_peak.md", "peak_int8_tops") or 4550.0
        bf16x2 = 2.0 * peaks["bf16_tflops"]
        qps = world * q_n * args.steps / (step_ms * 1e-3)
        e2e_qps = world * q_n * args.steps / (e2e_ms * 1e-3) if e2e_ms == e2e_ms else None
        traffic = _profile_value("exact2nn_u8fold_pair_10000x1M.md", "traffic_bytes_per_launch") if q_n == Q_N else None
        line = {
            "metric": METRIC,
            "value": round(qps, 1),
            "unit": "queries/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(step_ms / args.steps, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u8",
            "data": data_note,
            "config": {"workload": WORKLOAD if q_n == Q_N else WORKLOAD.replace("10,000", f"{q_n:,}"),
                       "queries_per_gpu": q_n, "base_rows": R_N, "dim": DIM,
                       "ratio": THRESHOLD, "l2_between_steps": "flushed (256 MiB write outside the timed events)",
                       "parallelism": f"query-sharded x{world}, base replicated"},
            "e2e": {"value": round(e2e_qps, 1) if e2e_qps else None, "unit": "queries/s",
                    "h2d_bytes_per_step": (q_n + R_N) * DIM, "d2h_bytes_per_step": q_n * 4,
                    "call": "cublas_2nn_sift(type=SIFT_U8_HOST) with pinned host buffers",
                    "h2d_copy_ms": round(h2d_ms, 4) if h2d_ms == h2d_ms else None,
                    "frac_of_h2d_copy": (round(h2d_ms / (e2e_ms / args.steps), 4)
                                         if h2d_ms == h2d_ms and e2e_ms == e2e_ms else None),
                    "h2d_note": "h2d_copy_ms: the step's input bytes copied alone from pinned memory on this box "
                                "(the PCIe bound of the call); frac = that / the call's time"},
            "gpu_launches": int(launches),
            "roofline": {"bound": "tensor", "kernel": "exact2nn_u8fold_pair_kernel", "achieved": round(achieved, 1),
                         "peak": round(peak_int8, 1), "unit": "TFLOP/s", "frac": round(achieved / peak_int8, 4),
                         "traffic": traffic,
                         "ops_per_launch": ops, "kernel_ms": round(kernel_ms, 4),
                         "peak_note": "dense int8 tcgen05 peak measured on this pool's B200 (int8 ops counted as 2 "
                                      "per MAC; MEASURED_PEAKS.json has no int8 figure)",
                         "frac_of_2x_bf16_" + peak_src: round(achieved / bf16x2, 4)},
            "clocks": clocks.summary(),
        }
        if args.truth_file:
            from matching_sift_b200 import vecs

            truth = vecs.read_ivecs(args.truth_file, count=q_n)
            line["recall_vs_truth"] = {
                "nn1_recall@1": round(vecs.recall_at(nn_idx[:, 0].cpu().numpy(), truth, 1), 6),
                "ratio_test_match_misses": vecs.recall_misses(matches.cpu().numpy().view(np.uint32), truth),
                "file": os.path.basename(args.truth_file)}
        if "pairs" in variants:
            v = variants["pairs"]
            pk_ms = v["step_ms"] / v["steps"]
            ach = v["ops"] / (pk_ms * 1e-3) / 1e12
            line.setdefault("variants", {})["pairs512"] = {
                "value": round(world * v["queries"] / (pk_ms * 1e-3), 1), "unit": "queries/s",
                "ms_per_step": round(pk_ms, 4), "steps": v["steps"], "dtype": "u8",
                "workload": f"{v['pairs']} image pairs, 500..8000 keypoints per side (log-uniform, seed 0), "
                            f"{v['queries']:,} query rows vs their pair's base rows, ratio test 0.8",
                "call": "sift_batch_plan_run: one CUDA graph (norms, records, one persistent "
                        "exact2nn_u8_pair_batch_kernel launch over the device work list, merge)",
                "inputs": "q + r = %.0f MB device-resident (> L2)" % (v["bytes"] / 1e6),
                "shape": v["shape"], "tuned_ms": v["tuned_ms"],
                "roofline": {"bound": "tensor", "achieved": round(ach, 1), "peak": round(peak_int8, 1),
                             "unit": "TFLOP/s", "frac": round(ach / peak_int8, 4), "ops_per_step": v["ops"],
                             "note": "whole graph time (4 launches: norms, records, search, merge), 2 ops per "
                                     "MAC"},
                "gpu_launches": v["launches"]}
        if "mutual" in variants:
            v = variants["mutual"]
            mu_ms = v["step_ms"] / v["steps"]
            line.setdefault("variants", {})["mutual512"] = {
                "value": round(world * v["rows"] / (mu_ms * 1e-3), 1), "unit": "queries/s",
                "ms_per_step": round(mu_ms, 4), "steps": v["steps"], "dtype": "u8",
                "workload": f"the {v['pairs']} image pairs of pairs512 matched both ways, {v['rows']:,} rows of the "
                            "first sets",
                "call": "sift2nn_match_mutual_batch + sift_compact_matches (two batched searches, cross-check, "
                        "per-pair match lists), preallocated outputs",
                "mutual_matches": v["mutual_matches"]}
        names = {"learned": "learned_hash", "lsh": "lsh", "cfg1": "cfg1_1000x10000", "float": "float32_general"}
        for key, name in names.items():
            if key in variants:
                v = dict(variants[key])
                v.pop("step_ms", None)
                v.pop("kernel_ms", None)
                line.setdefault("variants", {})[name] = v
        if "fp16" in variants:
            v = variants["fp16"]
            f16_peak = peaks["bf16_tflops"]
            ach = ops / (v["kernel_ms"] * 1e-3) / 1e12
            line.setdefault("variants", {})["fp16"] = {
                "value": round(world * q_n * v["steps"] / (v["step_ms"] * 1e-3), 1), "unit": "queries/s",
                "ms_per_step": round(v["step_ms"] / v["steps"], 4), "steps": v["steps"], "dtype": "f16",
                "call": "sift2nn_match(type=SIFT_HALF_DEVICE): FP16 rows searched in place by "
                        "exact2nn_f16_pair_kernel (kind::f16, f32 accumulation), same results as u8",
                "roofline": {"bound": "tensor", "kernel": "exact2nn_f16_pair_kernel", "achieved": round(ach, 1),
                             "peak": round(f16_peak, 1), "unit": "TFLOP/s", "frac": round(ach / f16_peak, 4),
                             "kernel_ms": round(v["kernel_ms"], 4),
                             "peak_note": f"dense bf16 cuBLAS ({peak_src}), the same tensor rate as f16"},
                "gpu_launches": v["launches"], "clocks": v["clocks"]}
        if not args.no_cpu_baseline:
            rate, sample, threads, kind = cpu_reference_rate(queries, base, 15.0)
            line["cpu_baseline"] = {"value": round(rate, 2), "unit": "queries/s", "cores": threads, "kind": kind,
                                    "sample": sample}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def fp16_leg(args, lib, ms, torch, qd, rd, flush, stream, q_n):
    """Device-resident timing of the FP16 kernel on the same rows as half."""
    import ctypes

    qh = qd.to(torch.float16)
    rh = rd.to(torch.float16)
    matches = torch.empty(q_n, dtype=torch.int32, device=qd.device)
    nn_idx = torch.empty((q_n, 2), dtype=torch.int32, device=qd.device)
    nn_dist = torch.empty((q_n, 2), dtype=torch.float32, device=qd.device)

    def step():
        rc = lib.sift2nn_match(qh.data_ptr(), rh.data_ptr(), ms.HALF_DEVICE, q_n, R_N, ms.METRIC_L2, THRESHOLD,
                               matches.data_ptr(), None, nn_idx.data_ptr(), nn_dist.data_ptr(), stream.cuda_stream)
        if rc != 0:
            raise ms.SiftError(rc, "sift2nn_match (FP16)")

    steps = max(3, args.steps // 2)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    launches0 = lib.sift_launch_count()
    lib.sift_profile_enable(1)
    with ClockSampler(qd.device.index or 0) as clocks:
        for k in range(steps):
            flush.fill_(k)
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    lib.sift_profile_enable(0)
    launches = lib.sift_launch_count() - launches0
    kt, kn = ctypes.c_double(0.0), ctypes.c_int(0)
    lib.sift_profile_collect(ctypes.byref(kt), ctypes.byref(kn))
    if ms.stream_status(stream.cuda_stream) != 0:
        raise RuntimeError("device status after FP16 steps")
    del qh, rh
    return {"step_ms": float(sum(a.elapsed_time(b) for a, b in ev)), "kernel_ms": kt.value / max(kn.value, 1),
            "steps": steps, "launches": int(launches), "clocks": clocks.summary(),
            "nn_idx": nn_idx}


def pairs_leg(args, ms, torch, dev, stream):
    """512 uneven image pairs (the batched workload) through a tuned batch plan."""
    from matching_sift_b200 import datagen

    data = datagen.make_pairs(512, seed=0)
    q = np.concatenate([a for a, _ in data])
    r = np.concatenate([b for _, b in data])
    pairs, off, ops = [], 0, 0
    for a, b in data:
        pairs.append([a.shape[0], b.shape[0], off])
        off += b.shape[0]
        ops += 2 * a.shape[0] * b.shape[0] * DIM
    qd, rd = torch.from_numpy(q).to(dev), torch.from_numpy(r).to(dev)
    plan = ms.BatchPlan(qd, rd, pairs, threshold=THRESHOLD, tune=True)
    info = plan.info()
    for _ in range(args.warmup):
        plan.run(stream)
    torch.cuda.synchronize()
    steps = max(3, args.steps)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = ms.lib().sift_launch_count()
    a.record(stream)
    for _ in range(steps):
        plan.run(stream)
    b.record(stream)
    torch.cuda.synchronize()
    if ms.stream_status(stream.cuda_stream) != 0:
        raise RuntimeError("device status after the batched steps")
    plan.close()
    return {"step_ms": a.elapsed_time(b), "steps": steps, "queries": int(q.shape[0]), "pairs": len(pairs),
            "ops": float(ops), "bytes": float(q.nbytes + r.nbytes),
            "shape": {"qpt": info["qpt"], "qbuf": info["qbuf"]},
            "tuned_ms": [round(x, 4) for x in info["tuned_ms"]],
            # graph replays are not counted by the library's launch counter; 4 kernels per replay
            "launches": int(ms.lib().sift_launch_count() - launches0) + 4 * steps}


def mutual_leg(args, ms, torch, dev, stream):
    """The 512 uneven image pairs matched both ways: sift2nn_match_mutual_batch
    (forward search with the ratio test, reverse search, cross-check) and
    sift_compact_matches (per-pair match lists for geometric verification),
    preallocated outputs, no host synchronisation inside the timed calls."""
    import ctypes

    from matching_sift_b200 import datagen

    data = datagen.make_pairs(512, seed=0)
    a = np.concatenate([x for x, _ in data])
    b = np.concatenate([y for _, y in data])
    pairs, off = [], 0
    for x, y in data:
        pairs.append([x.shape[0], y.shape[0], off])
        off += y.shape[0]
    pa = np.ascontiguousarray(np.asarray(pairs, dtype=np.uint32))
    ad, bd = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
    rows = a.shape[0]
    m = torch.empty(rows, dtype=torch.int32, device=dev)
    nn_idx = torch.empty((rows, 2), dtype=torch.int32, device=dev)
    nn_dist = torch.empty((rows, 2), dtype=torch.float32, device=dev)
    recs = torch.empty((rows, 5), dtype=torch.int32, device=dev)
    offs = torch.empty(len(pairs) + 1, dtype=torch.int32, device=dev)
    lib = ms.lib()
    pp = pa.ctypes.data_as(ctypes.c_void_p)

    def step():
        ms.check(lib.sift2nn_match_mutual_batch(ad.data_ptr(), bd.data_ptr(), b.shape[0], pp, len(pairs), THRESHOLD,
                                                m.data_ptr(), nn_idx.data_ptr(), nn_dist.data_ptr(),
                                                stream.cuda_stream), "sift2nn_match_mutual_batch")
        ms.check(lib.sift_compact_matches(m.data_ptr(), nn_dist.data_ptr(), rows, pp, len(pairs), recs.data_ptr(),
                                          rows, offs.data_ptr(), stream.cuda_stream), "sift_compact_matches")

    for _ in range(args.warmup):
        step()
    steps = max(3, args.steps)
    ms_call, _ = _time_calls(torch, stream, step, steps)
    if ms.stream_status(stream.cuda_stream) != 0:
        raise RuntimeError("device status after the mutual steps")
    return {"step_ms": ms_call * steps, "steps": steps, "rows": rows, "pairs": len(pairs),
            "mutual_matches": int(offs[-1].item())}


def _time_calls(torch, stream, fn, steps):
    """Mean device time (ms) of fn() over `steps` calls after one warm-up call."""
    fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        out = fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps, out


def _kernel_ms(lib, kind):
    """Mean device time (ms) of the kernels of one kind timed by the library since the last collection."""
    import ctypes

    t, n = ctypes.c_double(0.0), ctypes.c_int(0)
    lib.sift_profile_collect_kernel(kind, ctypes.byref(t), ctypes.byref(n))
    return t.value / n.value if n.value else None


def _search_points(ms, torch, stream, idx, qd, truth, copies, settings, steps, hbm, L, k):
    """Times idx.search at each (probes, min_candidates, max_dist) setting: queries/s,
    recall@1 (all queries, noisy-copy and fresh halves), candidates, and the
    hash / scan kernels' algorithmic bytes over their CUDA-event times."""
    lib = ms.lib()
    q_n = qd.shape[0]
    points = []
    for probes, min_cand, max_dist in settings:
        lib.sift_profile_enable(1)
        ms_call, out = _time_calls(torch, stream, lambda: idx.search(qd, probes=probes, min_candidates=min_cand,
                                                                     max_dist=max_dist, stream=stream), steps)
        lib.sift_profile_enable(0)
        hash_ms, scan_ms = _kernel_ms(lib, 1), _kernel_ms(lib, 2)
        _kernel_ms(lib, 0)
        got = out["nn_idx"][:, 0].cpu().numpy()
        hit = got == truth
        cand = float(out["candidates"].double().sum().item())
        # algorithmic bytes: query rows + codes (+ margins for probes) for the hash;
        # for the scan, query rows, two bucket bounds per probe and per compared
        # candidate its id (and code for k > 16) and its 128-byte row
        hash_bytes = q_n * 128 + L * q_n * 4 + (L * q_n * k * 4 if probes > 1 else 0)
        scan_bytes = q_n * 128 + L * probes * q_n * 8 + cand * (128 + (8 if k > 16 else 4))
        pt = {"probes": probes, "ms_per_call": round(ms_call, 4), "value": round(q_n / (ms_call * 1e-3), 1),
              "recall1": round(float(hit.mean()), 4), "recall1_copies": round(float(hit[copies].mean()), 4),
              "recall1_fresh": round(float(hit[~copies].mean()), 4),
              "candidates_mean": round(cand / q_n, 1)}
        if min_cand or max_dist:
            pt.update({"min_candidates": min_cand, "max_dist": max_dist,
                       "exact_fallback_queries": int(out["fallback"])})
        if hash_ms:
            pt["hash_kernel"] = {"ms": round(hash_ms, 4), "GB/s": round(hash_bytes / (hash_ms * 1e-3) / 1e9, 1),
                                 "frac_hbm": round(hash_bytes / (hash_ms * 1e-3) / 1e9 / hbm, 4)}
        if scan_ms:
            pt["scan_kernel"] = {"ms": round(scan_ms, 4), "GB/s": round(scan_bytes / (scan_ms * 1e-3) / 1e9, 1),
                                 "frac_hbm": round(scan_bytes / (scan_ms * 1e-3) / 1e9 / hbm, 4)}
        points.append(pt)
    return points


def _best_at(points, recall=0.8):
    ok = [p for p in points if p["recall1"] >= recall]
    return max(ok, key=lambda p: p["value"]) if ok else None


def learned_leg(args, ms, torch, dev, stream, qd, rd, base, truth, copies, hbm, lsh_grid):
    """Learned hash (MLP 128 -> 256 -> k, k in {16, 20, 24}) trained on 200,000
    generator queries labelled by the exact kernel; the base hashed and
    bucketed once per model (persistent index), then 2-NN of the bench queries
    at several operating points (probes, exact-fallback criteria) with
    recall@1 against the exact results, beside random-hyperplane LSH with the
    same bits, one table and the same probes."""
    from matching_sift_b200 import datagen

    tq = torch.from_numpy(datagen.make_queries(200_000, base, seed=7)).to(dev)
    steps = max(3, args.steps // 4)
    per_k = []
    for k in (16, 20, 24):
        t0 = time.perf_counter()
        model = ms.MlpHash.train(rd, tq, k=k, steps=1500, batch=2048, lr=2e-3, seed=1)
        train_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        idx = ms.HashIndex.mlp(rd, model)
        build_ms = (time.perf_counter() - t0) * 1e3
        settings = [(p, 0, 0.0) for p in (1, 4, 16, 64)] + [(16, 64, 0.0), (64, 64, 0.0), (16, 0, 30000.0),
                                                              (64, 0, 30000.0)]
        pts = _search_points(ms, torch, stream, idx, qd, truth, copies, settings, steps, hbm, 1, k)
        idx.close()
        lsh_same = [g for g in lsh_grid if g["k"] == k and g["L"] == 1]
        per_k.append({"k": k, "train_s": round(train_s, 2), "index_build_ms": round(build_ms, 2),
                      "best_at_recall_0.8": _best_at(pts), "points": pts,
                      "lsh_same_bits_L1": lsh_same[0]["points"] if lsh_same else None})
        del model
    best = [b for b in (x["best_at_recall_0.8"] for x in per_k) if b]
    top = max(best, key=lambda p: p["value"]) if best else None
    return {"value": top["value"] if top else None, "unit": "queries/s",
            "at": "fastest operating point with recall@1 >= 0.8 against the exact results over k in {16, 20, 24}",
            "operating_point": top,
            "workload": "same queries and base as the exact leg; persistent index (base hashed and bucketed once "
                        "per model); per call: query hash (tcgen05 MLP) + probe codes + candidate scan "
                        "[+ exact fallback]",
            "model": "MLP 128->256->k, BF16 weights, 1500 Adam steps x 2048 pairs, 200,000 training queries",
            "per_k": per_k}


def lsh_leg(args, ms, torch, dev, stream, qd, rd, truth, copies, hbm):
    """Random-hyperplane LSH over k in {12, 16, 20, 24} bits x L in {1, 2, 4, 8}
    tables (int8 hyperplanes = N(0,1) x 32 rounded, seed 1): the base hashed
    and bucketed once per configuration (persistent index), then searched with
    1 / 4 / 16 / 64 probes per table; recall@1 against the exact results,
    queries/s per call and the hash / scan kernels' achieved GB/s."""
    from matching_sift_b200 import datagen

    grid = []
    steps = 2
    for k in (12, 16, 20, 24):
        for L in (1, 2, 4, 8):
            planes = torch.from_numpy(datagen.quantize_planes(datagen.make_hyperplanes(k, L, seed=1))).to(dev)
            t0 = time.perf_counter()
            idx = ms.HashIndex.lsh(rd, planes)
            build_ms = (time.perf_counter() - t0) * 1e3
            pts = []
            for probes in (1, 4, 16, 64):
                pts += _search_points(ms, torch, stream, idx, qd, truth, copies, [(probes, 0, 0.0)], steps, hbm, L,
                                      k)
                if pts[-1]["recall1"] >= 0.95 or pts[-1]["ms_per_call"] > 150.0:
                    break
            idx.close()
            grid.append({"k": k, "L": L, "index_build_ms": round(build_ms, 2), "best_at_recall_0.8": _best_at(pts),
                         "points": pts})
    best = [g["best_at_recall_0.8"] | {"k": g["k"], "L": g["L"]} for g in grid if g["best_at_recall_0.8"]]
    top = max(best, key=lambda p: p["value"]) if best else None
    roof = None
    if top and "scan_kernel" in top:
        roof = {"bound": "hbm", "kernel": "lsh_scan_kernel", "achieved": top["scan_kernel"]["GB/s"], "peak": hbm,
                "unit": "GB/s", "frac": top["scan_kernel"]["frac_hbm"],
                "note": "algorithmic bytes (query rows, bucket bounds, per compared candidate its id and 128-byte "
                        "row) over the kernel's CUDA-event time at the fastest recall>=0.8 point"}
    return {"value": top["value"] if top else None, "unit": "queries/s", "operating_point": top,
            "at": "fastest (k, L, probes) with recall@1 >= 0.8 against the exact results",
            "call": "HashIndex.lsh / sift_index_search (base hashed and bucketed once per configuration)",
            "roofline": roof, "grid": grid}


def cfg1_leg(args, ms, torch, dev, stream):
    """The reference's small configuration: 1,000 queries x 10,000 base rows,
    u8 device rows (sift2nn_match) and float32 rows holding the integers
    (cublas_2nn_sift, type FLOAT_DEVICE, as the reference benchmark calls it)."""
    from matching_sift_b200 import datagen

    q, r = datagen.make_workload(1000, 10000, seed=1)
    qd, rd = torch.from_numpy(q).to(dev), torch.from_numpy(r).to(dev)
    qf, rf = qd.float(), rd.float()
    m = torch.empty(1000, dtype=torch.int32, device=dev)
    lib = ms.lib()
    steps = max(5, args.steps)
    u8_ms, _ = _time_calls(torch, stream, lambda: lib.sift2nn_match(qd.data_ptr(), rd.data_ptr(), ms.U8_DEVICE, 1000,
                                                                    10000, ms.METRIC_L2, THRESHOLD, m.data_ptr(),
                                                                    None, None, None, stream.cuda_stream), steps)
    f_ms, _ = _time_calls(torch, stream, lambda: lib.cublas_2nn_sift(qf.data_ptr(), rf.data_ptr(), ms.FLOAT_DEVICE,
                                                                     1000, 10000, m.data_ptr(), THRESHOLD, None, 1,
                                                                     0, 17), steps)
    return {"value": round(1000 / (u8_ms * 1e-3), 1), "unit": "queries/s", "ms_per_call": round(u8_ms, 4),
            "workload": "1,000 x 128 queries vs 10,000 x 128 base (seed 1), ratio test 0.8",
            "call": "sift2nn_match (u8 device rows)",
            "float32_call": {"ms_per_call": round(f_ms, 4), "value": round(1000 / (f_ms * 1e-3), 1),
                             "call": "cublas_2nn_sift(type=FLOAT_DEVICE) on float32 rows holding the integers "
                                     "(value check + u8 pack + search, synchronous)"}}


def float_leg(args, ms, torch, dev, stream, q_n, bf16_peak):
    """General float descriptors (the reference benchmark's default data:
    unit-normalised vectors of rand()-range values, src/helper.cu:40-58), 10,000
    x 1,000,000 float32: split FP16 rows, float keys (sift2nn_match FLOAT_DEVICE)."""
    lib = ms.lib()
    g = torch.Generator(device=dev)
    g.manual_seed(3)
    rf = torch.rand((R_N, DIM), device=dev, generator=g)
    rf /= rf.norm(dim=1, keepdim=True)
    qf = torch.rand((q_n, DIM), device=dev, generator=g)
    qf /= qf.norm(dim=1, keepdim=True)
    nn_idx = torch.empty((q_n, 2), dtype=torch.int32, device=dev)
    steps = max(3, args.steps // 4)
    lib.sift_profile_enable(1)
    ms_call, _ = _time_calls(torch, stream, lambda: lib.sift2nn_match(qf.data_ptr(), rf.data_ptr(), ms.FLOAT_DEVICE,
                                                                      q_n, R_N, ms.METRIC_L2, THRESHOLD, None, None,
                                                                      nn_idx.data_ptr(), None, stream.cuda_stream),
                             steps)
    lib.sift_profile_enable(0)
    k_ms = _kernel_ms(lib, 0)
    if ms.stream_status(stream.cuda_stream) != 0:
        raise RuntimeError("device status after the float steps")
    flops = 3 * 2.0 * q_n * R_N * DIM
    out = {"value": round(q_n / (ms_call * 1e-3), 1), "unit": "queries/s", "ms_per_call": round(ms_call, 4),
           "dtype": "f32 (split into FP16 hi + lo)",
           "workload": f"{q_n:,} x 128 float32 queries vs 1,000,000 x 128 float32 base, unit-normalised uniform "
                       "values (general floats: not integers)",
           "call": "sift2nn_match(type=SIFT_FLOAT_DEVICE): value check, split-FP16 pack, float norms, "
                   "exact2nn_float_pair_kernel (three kind::f16 products per tile), merge"}
    if k_ms:
        ach = flops / (k_ms * 1e-3) / 1e12
        out["roofline"] = {"bound": "tensor", "kernel": "exact2nn_float_pair_kernel", "kernel_ms": round(k_ms, 4),
                           "achieved": round(ach, 1), "peak": round(bf16_peak, 1), "unit": "TFLOP/s",
                           "frac": round(ach / bf16_peak, 4), "flops_per_launch": flops}
    del qf, rf
    return out


def reference_arm(args, world, rank):
    """The reference's own CPU implementation (host_brute) on all host threads, bounded samples."""
    if rank != 0:
        return
    import oracle
    from matching_sift_b200 import datagen

    base = datagen.make_base(R_N, seed=0)
    queries = datagen.make_queries(Q_N, base, seed=0)
    threads = _host_threads()
    kind = "reference" if oracle.ref_available() else "port"
    rf = np.ascontiguousarray(base, dtype=np.float32)

    def run(n, off):
        qs = queries[off:off + n]
        if kind == "reference":
            return oracle.ref_host_brute(qs.astype(np.float32), rf, nthreads=threads)
        return oracle.brute_2nn_u8(qs, base, nthreads=threads)

    # size one step to about 3 s of work
    t0 = time.perf_counter()
    run(threads, 0)
    per_q = (time.perf_counter() - t0) / threads
    n = max(threads, int(3.0 / max(per_q, 1e-9)) // threads * threads)
    n = min(n, Q_N)
    for k in range(args.warmup):
        run(n, (k * n) % (Q_N - n + 1))
    total = 0.0
    for k in range(args.steps):
        t0 = time.perf_counter()
        run(n, (k * n) % (Q_N - n + 1))
        total += time.perf_counter() - t0
    qps = n * args.steps / total
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(qps, 2),
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / args.steps, 2),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded generator standing in for ANN_SIFT1M)",
        "config": {"workload": WORKLOAD, "queries_per_step": n, "base_rows": R_N, "dim": DIM},
        "cpu_baseline": {"value": round(qps, 2), "unit": "queries/s", "cores": threads, "kind": kind,
                         "sample": f"{n} queries x {R_N} base rows per step"},
        "e2e": {"value": round(qps, 2), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
