#!/usr/bin/env python
"""Benchmark of the B200 Gaussian FIR path against the reference's CPU path.

Headline workload (one "step"): dip::Gauss FIR of a 256x256x256 uint16 volume (values uniform
0..4095, seeded), sigmas (1.5, 1.5, 3.0) in DIPlib order, truncation 3, boundary "mirror",
sfloat output -- run twice, with derivative orders (0,0,0) and (1,0,0).

  value  -- Gvoxel/s (output voxels of both runs / time) with inputs resident in HBM,
            CUDA-event timed over exactly K steps.  Input/output sets rotate over 4 copies
            (672 MB touched per rotation, > 126 MB L2), so every step reads cold data.
  e2e    -- the same metric through the public API with host buffers: per step a pinned
            host->device copy of the input, the two filter calls, and device->host copies of
            both outputs.
  roofline, cpu_baseline, clocks, gpu_launches -- see the keys below.

--impl reference times DIPlib's own OpenMP CPU implementation (oracle/_ref, built from the
unmodified reference sources) on the host cores instead.  Multi-GPU (torchrun): independent
replicas, one per GPU ("replicas only": the filter has no cross-GPU exchange).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gauss FIR Gvox/s, %HBM peak; batched & fwd+bwd vs plain, same GPU, ≤1e-5 err"
SHAPE = (256, 256, 256)           # numpy order (z, y, x)
SIGMAS = [1.5, 1.5, 3.0]          # DIPlib order (x, y, z)
ORDERS = ([0, 0, 0], [1, 0, 0])
BCS = ["mirror"]
TRUNC = 3.0
BYTES_PER_VOXEL = 2 + 4           # uint16 in, sfloat out
NSETS = 4                         # rotating input/output sets
CONFIG = {
    "workload": "dip::Gauss FIR 3D 256^3 uint16 -> sfloat, sigma (1.5,1.5,3.0), orders (0,0,0)+(1,0,0), "
                "truncation 3, mirror",
    "volume": "256x256x256", "dtype_in": "uint16", "dtype_out": "sfloat", "runs_per_step": 2,
    "l2": "inputs/outputs rotate over 4 sets (672 MB) > 126 MB L2",
}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def make_volume(seed=0):
    rng = np.random.default_rng(seed)
    return rng.integers(0, 4096, size=SHAPE, dtype=np.uint16)


def cpu_reference_step(x, threads):
    import oracle
    oracle.ref_set_threads(threads)
    for o in ORDERS:
        oracle.ref_gauss(x, SIGMAS, o, BCS, TRUNC)


def cpu_baseline(x, budget_s=12.0, max_reps=40):
    """The reference's OpenMP CPU path (or the oracle port if the reference was not built) on
    this host, timed on the full headline volume; min over repetitions, bounded by `budget_s`."""
    import oracle
    nvox = 2 * x.size
    if oracle.ref_available():
        cores = oracle.ref_set_threads(0)
        cpu_reference_step(x, 0)  # warm-up
        times = []
        t_end = time.perf_counter() + budget_s
        while len(times) < max_reps and (time.perf_counter() < t_end or len(times) < 2):
            t0 = time.perf_counter()
            cpu_reference_step(x, 0)
            times.append(time.perf_counter() - t0)
        return {"value": nvox / min(times) / 1e9, "unit": "Gvox/s", "cores": cores, "kind": "reference",
                "sample": f"full 256^3 step (both orders), min of {len(times)} reps, "
                          f"DIPlib sources built with -O3 -fopenmp, {cores} threads",
                "ms_per_step": min(times) * 1e3}
    # Oracle port: single thread on a z-slab sample of the volume.
    sl = x[:32]
    t0 = time.perf_counter()
    for o in ORDERS:
        oracle.gauss_fir(sl, SIGMAS, o, BCS, TRUNC)
    dt = time.perf_counter() - t0
    return {"value": 2 * sl.size / dt / 1e9, "unit": "Gvox/s", "cores": 1, "kind": "port",
            "sample": "32-plane slab of the volume, both orders, single-threaded C restatement"}


class ClockSampler:
    """Samples SM clocks and throttle reasons of one GPU with NVML while running."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

    def __init__(self, index):
        self.samples, self.reasons, self.stop_flag = [], set(), False
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None
        self.th = threading.Thread(target=self._run, daemon=True)

    def _sample(self):
        mhz = self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)
        r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        self.samples.append(mhz)
        for name, bit in self.REASONS.items():
            if r & bit:
                self.reasons.add(name)

    def _run(self):
        while not self.stop_flag:
            try:
                self._sample()
            except Exception:
                return
            time.sleep(0.002)

    def __enter__(self):
        if self.nv:
            self.th.start()
        return self

    def __exit__(self, *a):
        self.stop_flag = True
        if self.nv:
            self.th.join()
            try:
                self._sample()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def traffic_from_profiles():
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("fused3d_u16_256_bytes_per_launch")
    return None


def run_reference_arm(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    x = make_volume()
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libdipref.so was not built"}))
        return 0
    cores = oracle.ref_set_threads(0)
    for _ in range(args.warmup):
        cpu_reference_step(x, 0)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cpu_reference_step(x, 0)
    dt = time.perf_counter() - t0
    ms = dt / args.steps * 1e3
    value = 2 * x.size * args.steps / dt / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "Gvox/s", "impl": "reference", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform 0..4095)",
        "config": dict(CONFIG, parallelism="CPU, DIPlib OpenMP"),
        "cpu_baseline": {"value": value, "unit": "Gvox/s", "cores": cores, "kind": "reference",
                         "sample": f"full 256^3 step (both orders) x {args.steps}, {cores} threads"},
        "e2e": {"value": value, "unit": "Gvox/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_gpu_arm(args):
    import torch
    import torch.distributed as dist

    import diplib_b200 as dipcu

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    host = make_volume(seed=rank)
    xs = [torch.from_numpy(host.astype(np.int32)).to(dev).to(torch.uint16) for _ in range(NSETS)]
    for i in range(1, NSETS):
        xs[i] = (xs[i].to(torch.int32).add_(i) % 4096).to(torch.uint16)
    outs = [[torch.empty(SHAPE, dtype=torch.float32, device=dev) for _ in ORDERS] for _ in range(NSETS)]

    def call(s, j):
        dipcu.GaussFIR(xs[s], SIGMAS, ORDERS[j], BCS, TRUNC, out=outs[s][j])

    for i in range(args.warmup):
        for j in range(len(ORDERS)):
            call(i % NSETS, j)
    torch.cuda.synchronize()

    # One CUDA graph per (input set, order): each replays exactly one filter launch, so the host
    # keeps the GPU busy and the events below bracket device time only.
    graphs = {}
    for s in range(NSETS):
        for j in range(len(ORDERS)):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                call(s, j)
            graphs[s, j] = g
    for s in range(NSETS):
        for j in range(len(ORDERS)):
            graphs[s, j].replay()
    torch.cuda.synchronize()

    # Device-resident throughput: exactly K steps between two events; per-launch events give
    # the kernel's average duration for the roofline.
    kev = [[torch.cuda.Event(enable_timing=True) for _ in range(2 * len(ORDERS))] for _ in range(args.steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index if dev.index is not None else 0) as clk:
        stream = torch.cuda.current_stream(dev)
        start.record(stream)
        for i in range(args.steps):
            for j in range(len(ORDERS)):
                kev[i][2 * j].record(stream)
                graphs[i % NSETS, j].replay()
                kev[i][2 * j + 1].record(stream)
        stop.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms_total = start.elapsed_time(stop)
    kernel_ms = [kev[i][2 * j].elapsed_time(kev[i][2 * j + 1]) for i in range(args.steps) for j in range(len(ORDERS))]
    if world > 1:
        t = torch.tensor([ms_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    nvox = 2 * int(np.prod(SHAPE))
    value = world * nvox * args.steps / (ms_total * 1e-3) / 1e9
    del graphs

    # Host-side cost of one public-API call (no graph), for the record.
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(20):
        call(i % NSETS, i % len(ORDERS))
    host_call_us = (time.perf_counter() - t0) / 20 * 1e6
    torch.cuda.synchronize()

    # End to end through the public API with pinned host buffers.
    h_in = torch.from_numpy(host.astype(np.int32)).to(torch.uint16).pin_memory()
    h_out = [torch.empty(SHAPE, dtype=torch.float32).pin_memory() for _ in ORDERS]
    d_in = torch.empty(SHAPE, dtype=torch.uint16, device=dev)
    d_out = [torch.empty(SHAPE, dtype=torch.float32, device=dev) for _ in ORDERS]

    def e2e_step():
        d_in.copy_(h_in, non_blocking=True)
        for j, o in enumerate(ORDERS):
            dipcu.GaussFIR(d_in, SIGMAS, o, BCS, TRUNC, out=d_out[j])
            h_out[j].copy_(d_out[j], non_blocking=True)

    e2e_steps = max(3, min(args.steps, 20))
    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * nvox / (e2e_ms * 1e-3) / 1e9

    peak, peak_kind = load_peaks()
    avg_kernel_ms = sum(kernel_ms) / len(kernel_ms)
    achieved = BYTES_PER_VOXEL * int(np.prod(SHAPE)) / (avg_kernel_ms * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "Gvox/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform 0..4095)",
        "config": dict(CONFIG, parallelism=f"replicas x{world}" if world > 1 else "single GPU"),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic_from_profiles(), "peak_source": peak_kind,
                     "kernel": "fused3d_tma_kernel (TMA-pipelined z-marching tile kernel)", "bytes_per_voxel": BYTES_PER_VOXEL,
                     "avg_kernel_ms": avg_kernel_ms},
        "e2e": {"value": e2e_value, "unit": "Gvox/s", "h2d_bytes_per_step": int(h_in.numel() * 2),
                "d2h_bytes_per_step": int(sum(h.numel() * 4 for h in h_out)), "ms_per_step": e2e_ms},
        "clocks": clk.summary(),
        "host_us_per_call": host_call_us,
        "gpu_launches": args.steps * len(ORDERS),
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(host)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="dipcu", choices=["dipcu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
