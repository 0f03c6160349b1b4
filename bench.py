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
            both outputs, pipelined over three streams (upload, filters, download) with
            double-buffered device buffers.
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
    "graphs": "one CUDA graph per rotation of 4 steps (remainder steps one graph per launch)",
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


def cpu_model() -> str:
    """The host CPU's model name (/proc/cpuinfo), or the platform's processor string."""
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_baseline(x, budget_s=12.0, max_reps=40):
    """The reference's OpenMP CPU path (or the oracle port if the reference was not built) on
    this host, timed on the full headline volume; min over repetitions, bounded by `budget_s`.
    Also one thread (min of 2 reps) and the CPU model."""
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
        t1 = []
        for _ in range(2):
            t0 = time.perf_counter()
            cpu_reference_step(x, 1)
            t1.append(time.perf_counter() - t0)
        oracle.ref_set_threads(0)
        return {"value": nvox / min(times) / 1e9, "unit": "Gvox/s", "cores": cores, "kind": "reference",
                "sample": f"full 256^3 step (both orders), min of {len(times)} reps, "
                          f"DIPlib sources built with -O3 -fopenmp, {cores} threads",
                "ms_per_step": min(times) * 1e3, "cpu_model": cpu_model(), "host_cpus": os.cpu_count(),
                "value_1thread": nvox / min(t1) / 1e9, "ms_per_step_1thread": min(t1) * 1e3}
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


def read_overfetch_from_profiles(input_bytes):
    """DRAM bytes read per headline launch (ncu) over the input's bytes: the halo re-reads."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            r = json.load(f).get("fused3d_u16_256_read_bytes_per_launch")
        if r:
            return r / input_bytes
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
        "config": dict({k: v for k, v in CONFIG.items() if k != "graphs"}, parallelism="CPU, DIPlib OpenMP"),
        "cpu_baseline": {"value": value, "unit": "Gvox/s", "cores": cores, "kind": "reference",
                         "sample": f"full 256^3 step (both orders) x {args.steps}, {cores} threads",
                         "cpu_model": cpu_model()},
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
    n_launch0 = _launch_count()
    for s in range(NSETS):
        for j in range(len(ORDERS)):
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                call(s, j)
            graphs[s, j] = g
    launches_per_step = (_launch_count() - n_launch0) // NSETS   # a step replays one set's graphs
    # One graph of a whole rotation (the NSETS steps of sets 0 .. NSETS - 1, both orders each), so
    # that consecutive steps launch back to back.
    rot = _capture(lambda: [call(s, j) for s in range(NSETS) for j in range(len(ORDERS))])
    for s in range(NSETS):
        for j in range(len(ORDERS)):
            graphs[s, j].replay()
    rot.replay()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev)

    # Device-resident throughput: exactly K steps between two events (whole rotations, then the
    # remaining steps one graph each).  The launches run back to back, so the timed region over
    # its launches is the kernel's average launch duration (gaps between launches included).
    ms_total, clk = _timed_steps(rot, NSETS, [[graphs[s, j] for j in range(len(ORDERS))] for s in range(NSETS)],
                                 args.steps, dev)
    avg_kernel_ms = ms_total / (args.steps * launches_per_step)
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

    # End to end through the public API with pinned host buffers (pipelined: _e2e).
    h_in = torch.from_numpy(host.astype(np.int32)).to(torch.uint16).pin_memory()
    h_out = [torch.empty(SHAPE, dtype=torch.float32).pin_memory() for _ in ORDERS]
    d_in = [torch.empty(SHAPE, dtype=torch.uint16, device=dev) for _ in range(2)]
    d_out = [[torch.empty(SHAPE, dtype=torch.float32, device=dev) for _ in ORDERS] for _ in range(2)]

    def up(k):
        d_in[k].copy_(h_in, non_blocking=True)

    parts = [(lambda k, j=j: dipcu.GaussFIR(d_in[k], SIGMAS, ORDERS[j], BCS, TRUNC, out=d_out[k][j]),
              lambda k, j=j: h_out[j].copy_(d_out[k][j], non_blocking=True)) for j in range(len(ORDERS))]
    e2e = _e2e(up, parts, nvox, dev, world, h_in.numel() * 2, sum(h.numel() * 4 for h in h_out),
               steps=max(3, min(args.steps, 20)))

    peak, peak_kind = load_peaks()
    achieved = BYTES_PER_VOXEL * int(np.prod(SHAPE)) / (avg_kernel_ms * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "Gvox/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded uniform 0..4095)",
        "config": dict(CONFIG, parallelism=f"replicas x{world}" if world > 1 else "single GPU"),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic_from_profiles(), "peak_source": peak_kind,
                     "read_overfetch": read_overfetch_from_profiles(2 * int(np.prod(SHAPE))),
                     "kernel": "fused3d_ws_kernel (warp-specialised z-marching tile kernel)", "bytes_per_voxel": BYTES_PER_VOXEL,
                     "avg_kernel_ms": avg_kernel_ms},
        "e2e": e2e,
        "clocks": clk,
        "host_us_per_call": host_call_us,
        "gpu_launches": args.steps * launches_per_step,
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(host)
    del xs, outs, d_in, d_out
    torch.cuda.empty_cache()
    if not args.headline_only:
        line.update(other_workloads(args, achieved / peak))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def other_workloads(args, headline_frac):
    """The rest of the metric, measured in the same run: the plain 2D image, the batched uneven
    launch against the plain path, forward + backward against forward, and the structure tensor;
    each with its own roofline fraction (of the same measured peak), plus the three targets."""
    import argparse as _ap
    import torch
    sub = _ap.Namespace(**vars(args))
    sub.steps = max(10, min(args.steps, 20))
    out = {}
    sub2 = _ap.Namespace(**vars(args))
    sub2.steps = 64                          # two rotations of the 32 input sets, one graph each
    p2 = run_gauss2d(sub2, embedded=True)
    out["plain2d"] = {"workload": p2["config"]["workload"], "value": p2["value"], "unit": "Gvox/s",
                      "ms_per_step": p2["ms_per_step"], "frac": p2["roofline"]["frac"],
                      "kernel": p2["roofline"]["kernel"], "l2_flushed": p2["config"]["l2"],
                      "l2_resident_value": p2["l2_resident"]["value"]}
    torch.cuda.empty_cache()
    b = run_batch(sub, embedded=True)
    out["batched"] = {"workload": b["config"]["workload"], "value": b["value"], "unit": "Gvox/s",
                      "ms_per_run": b["ms_per_step"], "frac": b["roofline"]["frac"],
                      "vs_plain": b["vs_plain_large_image"]["ratio"],
                      "plain_large_image_gvox_s": b["vs_plain_large_image"]["plain_gvox_s"],
                      "plain_how": b["vs_plain_large_image"]["how"],
                      "vs_per_combination": b["vs_single_image"]["ratio"],
                      "per_combination_how": b["vs_single_image"]["how"],
                      "kernels_per_run": b["config"]["plan"]["kernels_per_run"]}
    torch.cuda.empty_cache()
    d = run_fwdbwd(sub, embedded=True)
    out["fwdbwd"] = {"workload": d["config"]["workload"], "fwd_ms": d["forward_only"]["ms_per_step"],
                     "fwdbwd_ms": d["ms_per_step"], "ratio": d["forward_only"]["fwd_plus_bwd_over_fwd"],
                     "value": d["value"], "unit": "Gvox/s", "frac": d["roofline"]["frac"],
                     "fwd_frac": d["forward_only"]["roofline"]["frac"]}
    torch.cuda.empty_cache()
    st = run_structure_tensor(sub, embedded=True)
    out["structure_tensor"] = {"workload": st["config"]["workload"], "value": st["value"], "unit": "Gvox/s",
                               "ms_per_step": st["ms_per_step"], "frac": st["roofline"]["frac"],
                               "fwd_plus_bwd_over_fwd": st["forward_only"]["fwd_plus_bwd_over_fwd"]}
    torch.cuda.empty_cache()
    out["targets"] = {
        "forward_ge_70pct_hbm": {"value": headline_frac, "met": headline_frac >= 0.70},
        "batched_ge_80pct_of_plain": {"value": out["batched"]["vs_plain"], "met": out["batched"]["vs_plain"] >= 0.80},
        "fwdbwd_le_2p5x_fwd": {"value": out["fwdbwd"]["ratio"], "met": out["fwdbwd"]["ratio"] <= 2.5},
    }
    return out


# ------------------------------------------------------------------------------------------------
# Further workloads (one JSON line each, same keys).  Selected with --workload; the default run
# above is the headline.  Each one rotates inputs/outputs over more than the 126 MB L2.
# ------------------------------------------------------------------------------------------------

def _device(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        if not dist.is_initialized():
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    return world, rank, dev


def _max_over_ranks(v: float, dev) -> float:
    """The largest `v` over all ranks of the process group (every rank takes this collective
    step), or `v` itself on one process."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(v)
    t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _launch_count() -> int:
    """Kernel launches libdipcu has issued (host side: a captured launch counts once, at capture)."""
    from diplib_b200 import _abi
    return int(_abi.lib().dipcu_launch_count())


def _capture(fn):
    import torch
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    return g


def _timed_steps(rot, nrot, singles, steps, dev):
    """Exactly `steps` steps between two events: steps // nrot replays of `rot` (one graph of the
    nrot steps of a rotation over the input sets 0 .. nrot - 1), then the remaining steps as
    the single-step graphs singles[i] (lists of graphs), starting again at set 0; barrier and
    synchronize on both sides, max over ranks.  Returns (total ms, clocks)."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    stream = torch.cuda.current_stream(dev)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index if dev.index is not None else 0) as clk:
        start.record(stream)
        for _ in range(steps // nrot):
            rot.replay()
        for i in range(steps % nrot):
            for g in singles[i]:
                g.replay()
        stop.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    total = _max_over_ranks(start.elapsed_time(stop), dev)
    return total, clk.summary()


def _timed(graph_lists, steps, dev):
    """Replays graph_lists[i % len] for `steps` steps between two events (barrier + sync on both
    sides, max over ranks).  Returns (total ms, per-step ms list, clocks)."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    stream = torch.cuda.current_stream(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index if dev.index is not None else 0) as clk:
        start.record(stream)
        for i in range(steps):
            ev[i][0].record(stream)
            for g in graph_lists[i % len(graph_lists)]:
                g.replay()
            ev[i][1].record(stream)
        stop.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    total = _max_over_ranks(start.elapsed_time(stop), dev)
    return total, [a.elapsed_time(b) for a, b in ev], clk.summary()


def _finish(line, world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if int(os.environ.get("RANK", "0")) == 0:
        print(json.dumps(line))
    return 0


def _base_line(args, world, value, ms_step, config, dtype="f32"):
    return {"metric": METRIC, "value": value, "unit": "Gvox/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype, "data": "synthetic (seeded)",
            "config": dict(config, parallelism=f"replicas x{world}" if world > 1 else "single GPU")}


def _ref_rate(fn, nvox, budget_s=8.0, max_reps=20):
    """(Gvox/s, cores, reps): the reference's OpenMP CPU path on `fn`, min over reps."""
    import oracle
    cores = oracle.ref_set_threads(0)
    fn()
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < max_reps and (time.perf_counter() < t_end or len(times) < 2):
        t0 = time.perf_counter()
        fn()
        times.append(time.perf_counter() - t0)
    return nvox / min(times) / 1e9, cores, len(times)


# ---- plain 2D (1024x1024 sfloat, sigma 2, order 0, mirror) ---------------------------------------

G2_SHAPE = (1024, 1024)
G2_CONFIG = {"workload": "dip::Gauss FIR 2D 1024^2 sfloat, sigma (2,2), order (0,0), truncation 3, mirror",
             "l2": "32 rotating input/output sets (268 MB) > 126 MB L2",
             "graphs": "one CUDA graph per rotation of 32 steps (remainder steps one graph each)"}


def run_gauss2d(args, embedded=False):
    import torch
    import diplib_b200 as dipcu
    world, rank, dev = _device(args)
    nsets = 32
    rng = np.random.default_rng(10 + rank)
    host = rng.random(G2_SHAPE, dtype=np.float32)
    xs = [torch.from_numpy(host).to(dev).add_(i * 1e-3) for i in range(nsets)]
    ys = [torch.empty(G2_SHAPE, dtype=torch.float32, device=dev) for _ in range(nsets)]

    def call(i):
        dipcu.GaussFIR(xs[i], [2.0, 2.0], [0, 0], ["mirror"], 3.0, out=ys[i])

    for i in range(max(args.warmup, nsets)):
        call(i % nsets)
    graphs = [[_capture(lambda i=i: call(i))] for i in range(nsets)]
    rot = _capture(lambda: [call(i) for i in range(nsets)])    # a rotation over the sets, one graph
    for gl in graphs:
        gl[0].replay()
    rot.replay()
    total, clk = _timed_steps(rot, nsets, graphs, args.steps, dev)
    npx = int(np.prod(G2_SHAPE))
    value = world * npx * args.steps / (total * 1e-3) / 1e9
    avg = total / args.steps                                    # one launch per step, back to back
    peak, kind = load_peaks()
    line = _base_line(args, world, value, total / args.steps, G2_CONFIG)
    ach = 8 * npx / (avg * 1e-3) / 1e9
    line["roofline"] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                        "traffic": None, "peak_source": kind, "kernel": "fused2d_ws_kernel (warp per tile)", "bytes_per_voxel": 8,
                        "avg_kernel_ms": avg}
    line["clocks"] = clk
    line["gpu_launches"] = args.steps
    # L2-resident: the same input and output every step (8 MB working set stays in the 126 MB L2).
    same = _capture(lambda: [call(0) for _ in range(nsets)])
    same.replay()
    t_res, _ = _timed_steps(same, nsets, [graphs[0]] * nsets, args.steps, dev)
    line["l2_resident"] = {"value": world * npx * args.steps / (t_res * 1e-3) / 1e9, "unit": "Gvox/s",
                           "ms_per_step": t_res / args.steps,
                           "how": "one input/output set replayed back to back (8 MB, stays in L2)"}
    if embedded:
        return line
    # e2e: pinned host image in, result out.
    h_in = torch.from_numpy(host).pin_memory()
    h_out = torch.empty(G2_SHAPE, dtype=torch.float32).pin_memory()
    d_in = [torch.empty_like(xs[0]) for _ in range(2)]
    d_out = [torch.empty_like(ys[0]) for _ in range(2)]
    line["e2e"] = _e2e(lambda k: d_in[k].copy_(h_in, non_blocking=True),
                       [(lambda k: dipcu.GaussFIR(d_in[k], [2.0, 2.0], [0, 0], ["mirror"], 3.0, out=d_out[k]),
                         lambda k: h_out.copy_(d_out[k], non_blocking=True))], npx, dev, world, 4 * npx, 4 * npx)
    if rank == 0 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            v, cores, reps = _ref_rate(lambda: oracle.ref_gauss(host, [2.0, 2.0], [0, 0], ["mirror"], 3.0), npx)
            line["cpu_baseline"] = {"value": v, "unit": "Gvox/s", "cores": cores, "kind": "reference",
                                    "sample": f"full 1024^2 image, min of {reps} reps"}
    return _finish(line, world)


def _e2e(up, parts, nvox, dev, world, h2d, d2h, steps=20):
    """End-to-end throughput through the public API, pipelined the way a caller streaming data
    runs it: every step uploads its inputs from pinned host memory (copy stream), runs its work
    (compute stream) and downloads its results (copy-back stream).  up(k) and each (work, down)
    pair of `parts` issue the step's pieces for device buffer set k (two sets, alternating) on the
    current stream; a part's download waits for that part's work only.  So step i's work overlaps
    step i + 1's upload and step i - 1's download.  Every step still moves its own inputs up and
    results down inside the timed region."""
    import torch
    main = torch.cuda.current_stream(dev)
    st = [torch.cuda.Stream(dev) for _ in range(3)]
    ev_up = [torch.cuda.Event() for _ in range(2)]
    ev_work = [[torch.cuda.Event() for _ in range(2)] for _ in parts]
    ev_down = [torch.cuda.Event() for _ in range(2)]

    def step(i):
        k = i % 2
        st[0].wait_event(ev_work[-1][k])            # set k's previous work has read its inputs
        with torch.cuda.stream(st[0]):
            up(k)
        ev_up[k].record(st[0])
        st[1].wait_event(ev_up[k])
        st[1].wait_event(ev_down[k])                # set k's previous results are downloaded
        for j, (work, down) in enumerate(parts):
            with torch.cuda.stream(st[1]):
                work(k)
            ev_work[j][k].record(st[1])
            st[2].wait_event(ev_work[j][k])
            with torch.cuda.stream(st[2]):
                down(k)
        ev_down[k].record(st[2])

    def run(n):
        for s_ in st:
            s_.wait_stream(main)
        for i in range(n):
            step(i)
        for s_ in st:
            main.wait_stream(s_)

    run(2)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(main)
    run(steps)
    e1.record(main)
    torch.cuda.synchronize()
    ms = _max_over_ranks(e0.elapsed_time(e1) / steps, dev)
    return {"value": world * nvox / (ms * 1e-3) / 1e9, "unit": "Gvox/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "ms_per_step": ms,
            "pipelining": "uploads, work and downloads on three streams, two device buffer sets"}


# ---- batched uneven 2D (512 images) --------------------------------------------------------------

B_SIGMAS = [0.8, 1.0, 2.0, 4.0, 8.0]
B_BCS = ["mirror", "periodic", "add zeros"]
B_CONFIG = {"workload": "batched dip::GaussFIR: 512 2D sfloat images, sides uniform 64..2048, sigma from "
                        "{0.8,1,2,4,8} per image, order per axis from {0,1,2}, boundary from {mirror, periodic, "
                        "add zeros}, truncation 3; the weights kernel and one persistent row-march launch over a "
                        "device work queue, replayed as one CUDA graph, row runs autotuned per y half-width",
            "l2": "the batch holds 2.3 GB of input and 2.3 GB of output (> 126 MB L2)"}


def make_batch_params(seed=0, n=512):
    rng = np.random.default_rng(seed)
    shapes, params = [], []
    for _ in range(n):
        h, w = (int(v) for v in rng.integers(64, 2049, 2))
        shapes.append((h, w))
        params.append((float(rng.choice(B_SIGMAS)), [int(rng.integers(0, 3)), int(rng.integers(0, 3))],
                       str(rng.choice(B_BCS))))
    return shapes, params


def run_batch(args, embedded=False):
    import torch
    import diplib_b200 as dipcu
    from diplib_b200.batch import BatchPlan
    world, rank, dev = _device(args)
    shapes, params = make_batch_params(seed=rank)
    gen = torch.Generator(device=dev).manual_seed(20 + rank)
    ins = [torch.rand(s, generator=gen, device=dev) for s in shapes]
    outs = [torch.empty(s, device=dev) for s in shapes]
    plan = BatchPlan(ins, outs, [p[0] for p in params], [p[1] for p in params], [p[2] for p in params],
                     graph=True, autotune=True)
    for _ in range(args.warmup):
        plan.run()
    torch.cuda.synchronize()

    class _G:
        def replay(self):
            plan.run()

    total, per, clk = _timed([[_G()]], args.steps, dev)
    npx = sum(h * w for h, w in shapes)
    value = world * npx * args.steps / (total * 1e-3) / 1e9
    avg = sum(per) / len(per)
    peak, kind = load_peaks()
    line = _base_line(args, world, value, total / args.steps, B_CONFIG)
    line["config"]["plan"] = plan.info()
    ach = 8 * npx / (avg * 1e-3) / 1e9
    line["roofline"] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                        "traffic": None, "peak_source": kind, "kernel": "whole batch run (weights + the persistent row-march launch)",
                        "bytes_per_voxel": 8, "avg_kernel_ms": avg}
    line["clocks"] = clk
    line["gpu_launches"] = plan.info()["kernels_per_run"] * args.steps   # all kernels of the captured graph
    # The same per-pixel work as single large images: per (sigma, orders, boundary condition)
    # combination of the batch, the plain path's rate on one 4096x4096 image; the batch's pixel
    # shares weight them.
    share = {}
    for (h, w), (sg, o, bc) in zip(shapes, params):
        key = (sg, o[0], o[1], bc)
        share[key] = share.get(key, 0) + h * w
    big = torch.rand((4096, 4096), generator=gen, device=dev)
    bigs = [big, big.clone().add_(1e-3)]
    bigo = [torch.empty_like(big) for _ in range(2)]
    t_single = 0.0
    rates = {}
    for key, px in sorted(share.items()):
        sg, ox, oy, bc = key
        gl = [[_capture(lambda i=i: dipcu.GaussFIR(bigs[i], [sg, sg], [ox, oy], [bc], 3.0, out=bigo[i]))]
              for i in range(2)]
        for g in gl:
            g[0].replay()
        tt, _, _ = _timed(gl, 10, dev)
        r = 4096 * 4096 * 10 / (tt * 1e-3) / 1e9
        rates[f"s{sg}_o{ox}{oy}_{bc.replace(' ', '')}"] = round(r, 2)
        t_single += px / (r * 1e9)
    single_rate = npx / t_single / 1e9
    line["vs_single_image"] = {"single_image_gvox_s": single_rate, "ratio": value / world / single_rate,
                               "how": "plain dipcu_gauss_fir on one 4096^2 image per (sigma, orders, boundary "
                                      "condition) combination, weighted by the batch's pixel shares", "rates": rates}
    # The plain 2D tile kernel's large-image rate: one 4096^2 image, sigma 2, order (0,0), mirror.
    gl = [[_capture(lambda i=i: dipcu.GaussFIR(bigs[i], [2.0, 2.0], [0, 0], ["mirror"], 3.0, out=bigo[i]))]
          for i in range(2)]
    for g in gl:
        g[0].replay()
    tt, _, _ = _timed(gl, 10, dev)
    plain_rate = 4096 * 4096 * 10 / (tt * 1e-3) / 1e9
    line["vs_plain_large_image"] = {"plain_gvox_s": plain_rate, "ratio": value / world / plain_rate,
                                    "how": "plain dipcu_gauss_fir on one 4096^2 sfloat image, sigma 2, order (0,0), "
                                           "mirror (the 2D tile kernel's large-image rate)"}
    if embedded:
        plan.close()
        return line
    # e2e: every image in from pinned host memory, every result back; a second plan over a second
    # set of device buffers for the pipelined steps.
    h_in = [t.cpu().pin_memory() for t in ins]
    h_out = [torch.empty(s).pin_memory() for s in shapes]
    ins2 = [t.clone() for t in ins]
    outs2 = [torch.empty_like(t) for t in outs]
    plan2 = BatchPlan(ins2, outs2, [p[0] for p in params], [p[1] for p in params], [p[2] for p in params],
                      graph=True, autotune=True)
    sets = [(plan, ins, outs), (plan2, ins2, outs2)]

    def up(k):
        for a, b in zip(h_in, sets[k][1]):
            b.copy_(a, non_blocking=True)

    def down(k):
        for a, b in zip(h_out, sets[k][2]):
            a.copy_(b, non_blocking=True)

    line["e2e"] = _e2e(up, [(lambda k: sets[k][0].run(), down)], npx, dev, world, 4 * npx, 4 * npx, steps=5)
    if rank == 0 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            hs = [t.cpu().numpy() for t in ins[:24]]
            sample_px = sum(a.size for a in hs)

            def ref():
                for a, (sg, o, bc) in zip(hs, params[:24]):
                    oracle.ref_gauss(a, [sg, sg], o, [bc], 3.0)

            v, cores, reps = _ref_rate(ref, sample_px)
            line["cpu_baseline"] = {"value": v, "unit": "Gvox/s", "cores": cores, "kind": "reference",
                                    "sample": f"the first 24 images of the batch ({sample_px / 1e6:.1f} Mpx), "
                                              f"min of {reps} reps"}
    plan.close()
    return _finish(line, world)


# ---- differentiable 2D Gaussian (2048x2048, sigma 3, four orders, forward + backward) -------------

D_SHAPE = (2048, 2048)
D_ORDERS = [(0, 0), (1, 0), (0, 1), (2, 0)]
D_CONFIG = {"workload": "differentiable dip::GaussFIR 2D 2048^2 sfloat, sigma 3, orders (0,0),(1,0),(0,1),(2,0), "
                        "mirror; step = forward + backward (input and sigma gradients) of all four",
            "l2": "4 rotating sets of input, upstream gradient, output and gradients (268 MB) > 126 MB L2"}


def run_fwdbwd(args, embedded=False):
    import torch
    import diplib_b200 as dipcu
    from diplib_b200 import torch_ops
    world, rank, dev = _device(args)
    nsets = 4
    gen = torch.Generator(device=dev).manual_seed(30 + rank)
    xs = [torch.rand(D_SHAPE, generator=gen, device=dev) for _ in range(nsets)]
    gys = [torch.randn(D_SHAPE, generator=gen, device=dev) for _ in range(nsets)]
    ys = [torch.empty(D_SHAPE, device=dev) for _ in range(nsets)]
    gxs = [torch.empty(D_SHAPE, device=dev) for _ in range(nsets)]
    gss = [torch.empty(2, dtype=torch.float64, device=dev) for _ in range(nsets)]

    def fwd(i, o):
        dipcu.GaussFIR(xs[i], [3.0, 3.0], list(o), ["mirror"], 3.0, out=ys[i])

    def bwd(i, o):
        gx, gs = torch_ops.gauss_backward(gys[i], xs[i], [3.0, 3.0], list(o), ["mirror"], 3.0, True, True)
        gxs[i].copy_(gx)
        gss[i].copy_(gs)

    def bwd_raw(i, o):
        import ctypes
        from diplib_b200 import _abi
        d_go, d_x, d_gx = dipcu.image_desc(gys[i]), dipcu.image_desc(xs[i]), dipcu.image_desc(gxs[i])
        dipcu.filtering.check(_abi.lib().dipcu_gauss_fir_backward(
            ctypes.byref(d_go), ctypes.byref(d_x), ctypes.byref(d_gx), ctypes.c_void_p(gss[i].data_ptr()),
            (ctypes.c_double * 2)(3.0, 3.0), (ctypes.c_uint32 * 2)(*o), (ctypes.c_int32 * 2)(0, 0), 3.0,
            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))

    for i in range(nsets):
        for o in D_ORDERS:
            fwd(i, o)
            bwd(i, o)
    torch.cuda.synchronize()
    g_f = [[_capture(lambda i=i, o=o: fwd(i, o)) for o in D_ORDERS] for i in range(nsets)]
    n0 = _launch_count()
    g_fb = [[_capture(lambda i=i, o=o: (fwd(i, o), bwd_raw(i, o))) for o in D_ORDERS] for i in range(nsets)]
    launches_per_step = (_launch_count() - n0) // nsets     # a step replays one set's graphs
    for gl in g_f + g_fb:
        for g in gl:
            g.replay()
    t_f, per_f, _ = _timed(g_f, args.steps, dev)
    t_fb, per_fb, clk = _timed(g_fb, args.steps, dev)
    npx = int(np.prod(D_SHAPE)) * len(D_ORDERS)
    value = world * npx * args.steps / (t_fb * 1e-3) / 1e9
    peak, kind = load_peaks()
    line = _base_line(args, world, value, t_fb / args.steps, D_CONFIG)
    ach = 20 * npx / (t_fb / args.steps * 1e-3) / 1e9
    line["roofline"] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                        "traffic": None, "peak_source": kind, "kernel": "whole step (forward 8 B + backward 12 B "
                        "per pixel and order)", "bytes_per_voxel": 20, "avg_kernel_ms": t_fb / args.steps}
    line["forward_only"] = {"ms_per_step": t_f / args.steps, "gvox_s": world * npx * args.steps / (t_f * 1e-3) / 1e9,
                            "fwd_plus_bwd_over_fwd": t_fb / t_f}
    ach_f = 8 * npx / (t_f / args.steps * 1e-3) / 1e9
    line["forward_only"]["roofline"] = {"achieved": ach_f, "peak": peak, "unit": "GB/s", "frac": ach_f / peak,
                                        "bytes_per_voxel": 8}
    line["clocks"] = clk
    line["gpu_launches"] = launches_per_step * args.steps
    if embedded:
        return line
    if rank == 0 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            hx = xs[0].cpu().numpy()

            def ref():
                for o in D_ORDERS:
                    oracle.ref_gauss(hx, [3.0, 3.0], list(o), ["mirror"], 3.0)

            v, cores, reps = _ref_rate(ref, npx)
            line["cpu_baseline"] = {"value": v, "unit": "Gvox/s", "cores": cores, "kind": "reference",
                                    "sample": f"forward only (DIPlib has no backward): the four orders on one "
                                              f"2048^2 image, min of {reps} reps"}
    return _finish(line, world)


# ---- differentiable structure tensor (8 x 192^3, forward + backward) ------------------------------

S_SHAPE = (192, 192, 192)
S_BATCH = 8
S_CONFIG = {"workload": "differentiable dip::StructureTensor, 8 sfloat volumes of 192^3 (Gauss sigma 2 of N(0,1)), "
                        "gradient sigma 1, tensor sigma 4, mirror; loss = sum of the 6 components times N(0,1) "
                        "weights; step = forward + backward w.r.t. the input of all 8 (gradient images recomputed)",
            "l2": "8 volumes with 6-component tensors and weights (2.9 GB) > 126 MB L2"}


def run_structure_tensor(args, embedded=False):
    import torch
    from diplib_b200 import torch_ops
    world, rank, dev = _device(args)
    gen = torch.Generator(device=dev).manual_seed(40 + rank)
    import diplib_b200 as dipcu
    xs = []
    for _ in range(S_BATCH):
        n = torch.randn(S_SHAPE, generator=gen, device=dev)
        xs.append(dipcu.GaussFIR(n, 2.0, 0, "mirror", 3.0))
    ws = [torch.randn((6,) + S_SHAPE, generator=gen, device=dev) for _ in range(S_BATCH)]
    ts = [None] * S_BATCH
    gxs = [None] * S_BATCH

    def fwd(i):
        ts[i] = torch_ops.structure_tensor(xs[i], 1.0, 4.0, "mirror", 3.0)

    def fb(i):
        ts[i] = torch_ops.structure_tensor(xs[i], 1.0, 4.0, "mirror", 3.0)
        gxs[i] = torch_ops.structure_tensor_backward(ws[i], xs[i], 1.0, 4.0, "mirror", 3.0)

    for i in range(S_BATCH):
        fb(i)
    torch.cuda.synchronize()
    g_f = [[_capture(lambda i=i: fwd(i)) for i in range(S_BATCH)]]
    n0 = _launch_count()
    g_fb = [[_capture(lambda i=i: fb(i)) for i in range(S_BATCH)]]
    launches_per_step = _launch_count() - n0               # a step replays all eight graphs
    for gl in g_f + g_fb:
        for g in gl:
            g.replay()
    t_f, _, _ = _timed(g_f, max(3, args.steps // 10), dev)
    steps = max(3, args.steps // 10)
    t_fb, _, clk = _timed(g_fb, steps, dev)
    nvox = S_BATCH * int(np.prod(S_SHAPE))
    value = world * nvox * steps / (t_fb * 1e-3) / 1e9
    peak, kind = load_peaks()
    args_steps = args.steps
    args.steps = steps
    line = _base_line(args, world, value, t_fb / steps, S_CONFIG)
    args.steps = args_steps
    ach = 60 * nvox / (t_fb / steps * 1e-3) / 1e9
    line["roofline"] = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                        "traffic": None, "peak_source": kind, "kernel": "whole step (forward 28 B + backward 32 B "
                        "per voxel)", "bytes_per_voxel": 60, "avg_kernel_ms": t_fb / steps}
    line["forward_only"] = {"ms_per_step": t_f / steps, "gvox_s": world * nvox * steps / (t_f * 1e-3) / 1e9,
                            "fwd_plus_bwd_over_fwd": t_fb / t_f}
    line["clocks"] = clk
    line["gpu_launches"] = launches_per_step * steps
    if embedded:
        return line
    if rank == 0 and not args.no_cpu_baseline:
        import oracle
        if oracle.ref_available():
            hx = xs[0].cpu().numpy()
            v, cores, reps = _ref_rate(lambda: oracle.ref_structure_tensor(hx, 1.0, 4.0, "mirror", 3.0),
                                       hx.size, budget_s=10.0, max_reps=5)
            line["cpu_baseline"] = {"value": v, "unit": "Gvox/s", "cores": cores, "kind": "reference",
                                    "sample": f"forward only (DIPlib has no backward): one 192^3 volume, "
                                              f"min of {reps} reps"}
    return _finish(line, world)


WORKLOADS = {"gauss2d": run_gauss2d, "batch": run_batch, "fwdbwd": run_fwdbwd,
             "structure_tensor": run_structure_tensor}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="dipcu", choices=["dipcu", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true",
                    help="the headline workload alone, without the other configurations' summaries")
    ap.add_argument("--workload", default="gauss3d", choices=["gauss3d"] + sorted(WORKLOADS),
                    help="gauss3d: the headline 256^3 uint16 volume (default); the others are the further "
                         "configurations (plain 2D, batched uneven 2D, differentiable 2D, structure tensor)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload != "gauss3d":
        return WORKLOADS[args.workload](args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
