#!/usr/bin/env python
"""Benchmark of the escape-time hot path (G iterations per second).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step renders one frame of the workload.  Rank 0 prints one JSON line:
  value   device-resident throughput: the frame's device passes on inputs
          already in HBM, CUDA-event timed per step with an L2 flush
          (a 512 MiB write) between steps, max over ranks;
  e2e     the same metric through engine.render_frame_ssaa with host
          buffers: host planning, H2D of the step's inputs and D2H of the
          RGB frame inside the timed region;
  roofline, clocks, cpu_baseline, gpu_launches as documented in DESIGN.md.
Multi-GPU: one process per GPU, every rank renders its own frame (weak
scaling, no collective on the data path).
"""
import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time
from datetime import timedelta
from decimal import Decimal

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FP64_FLOPS_PER_ITER = 8.0  # Mandelbrot FP64 step: 3 mul + 1 fma (2) + 3 add/sub


# --------------------------------------------------------------- workloads
def workload_cfg1():
    """640x360 Mandelbrot, FP64 direct, centre (-0.65, 0), width 4, max_iter 1000,
    histogram-equalised colouring, 1x SSAA."""
    return dict(name="mandelbrot_fp64_640x360_hist", W=640, H=360, max_iter=1000, cx="-0.65",
                cy="0.0", width="4.0", scheme=11, factor=1, fractal_type=0,
                precision_mode="1e-12 (FP64)", flops_per_iter=FP64_FLOPS_PER_ITER,
                bound="fp64")


WORKLOADS = {"cfg1": workload_cfg1}
DEFAULT_WORKLOAD = "cfg1"


# ------------------------------------------------------------------ helpers
def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def fma_peak_tflops(precision, stream_h, torch):
    """Dependent-FMA probe of the FP64/FP32 vector pipe (TFLOP/s, best of 5)."""
    from fractura_b200 import _lib
    L = _lib.load()
    blocks = 148 * 16
    scratch = torch.empty(blocks, dtype=torch.float64, device="cuda")
    flops = C.c_double()
    iters = 4096 if precision == 64 else 16384
    best = 0.0
    st = torch.cuda.current_stream()
    for rep in range(6):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        _lib.check(L.ap_fma_peak_launch(precision, blocks, iters, C.c_void_p(scratch.data_ptr()),
                                        C.byref(flops), C.c_void_p(st.cuda_stream)), "ap_fma_peak_launch")
        b.record(st)
        b.synchronize()
        if rep > 0:
            best = max(best, flops.value / (a.elapsed_time(b) * 1e-3) / 1e12)
    return best


def load_traffic(workload_name):
    path = os.path.join(ROOT, "profiles", f"{workload_name}.traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return None


# --------------------------------------------------------- reference arm
def cpu_reference_arm(args, wl, rank, world):
    """The reference's CPU path of the hot loop, restated in C (oracle/), on all host cores."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    value, sample = time_oracle(wl, args.steps, args.warmup)
    line = {"metric": "G iter/s", "value": value, "unit": "G iter/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": config_of(wl, args),
            "cpu_baseline": {"value": value, "unit": "G iter/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "G iter/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def time_oracle(wl, steps, warmup, rows=None):
    """Time the oracle on the workload frame (or every n-th row); returns (G iter/s, description)."""
    import oracle
    from fractura_b200 import abi
    from helpers import direct_params
    m = dict(W=wl["W"], H=wl["H"], factor=wl["factor"], max_iter=wl["max_iter"], cx=wl["cx"],
             cy=wl["cy"], width=wl["width"], scheme=wl["scheme"], fractal_type=wl["fractal_type"])
    p = direct_params(m, abi.AP_TIER_FP64, abi.AP_ARITH_REF_CPU)
    p.flags = abi.AP_FLAG_NO_RGB
    fr = oracle.Frame(wl["W"], wl["H"])
    times = []
    for it in range(warmup + steps):
        t0 = time.perf_counter()
        oracle.render_pass(p, fr)
        oracle.histogram_cdf(fr, wl["max_iter"])
        times.append(time.perf_counter() - t0)
    iters = nominal_iterations(fr.kmap, wl["max_iter"])
    t = float(np.mean(times[warmup:]))
    return iters / t / 1e9, f"full {wl['W']}x{wl['H']} frame, oracle C port, mean of {steps} steps"


def nominal_iterations(kmap, max_iter):
    """Sum of escape steps, max_iter for never-escaped samples, 0 for cardioid skips."""
    k = np.asarray(kmap)
    return float(k[k >= 0].astype(np.int64).sum() + np.int64(max_iter) * np.count_nonzero(k == -1))


def config_of(wl, args):
    return {"workload": wl["name"], "width": wl["W"], "height": wl["H"], "max_iter": wl["max_iter"],
            "ssaa": wl["factor"], "precision_mode": wl["precision_mode"],
            "l2": "flushed between timed steps (512 MiB write)",
            "parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "single"}


# -------------------------------------------------------------- our arm
def our_arm(args, wl, rank, world, local_rank):
    import torch
    from fractura_b200 import _lib, abi, engine

    torch.cuda.set_device(local_rank)
    dev_stream = torch.cuda.Stream()
    stream_h = C.c_void_p(dev_stream.cuda_stream)
    W, H = wl["W"], wl["H"]
    view = engine.plan_direct_view(W, H, wl["factor"], Decimal(wl["cx"]), Decimal(wl["cy"]),
                                   Decimal(wl["width"]), abi.AP_TIER_FP64)
    num_bins = 65536 if wl["scheme"] == 11 else 2048
    with torch.cuda.stream(dev_stream):
        fr = engine._DeviceFrame(W, H, False, slot=0)
        lut = engine.get_device_lut(None)
        kmap = torch.empty((H, W), dtype=torch.int32, device="cuda")
        flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    def params():
        p = abi.new_params(width=W, height=H, factor=wl["factor"], max_iter=wl["max_iter"],
                           fractal_type=wl["fractal_type"], tier=abi.AP_TIER_FP64,
                           arith=abi.AP_ARITH_REF_CPU, scheme_id=wl["scheme"], num_bins=num_bins)
        for k, v in view.items():
            setattr(p, k, v)
        return p

    L = _lib.load()
    pass_events = []

    def device_step(record):
        """The frame's device passes (what render_frame issues after planning)."""
        p = params()
        p.flags = abi.AP_FLAG_NO_RGB
        b = engine._buffers(fr, lut, kmap=kmap)
        if record:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(dev_stream)
        _lib.check(L.ap_render_pass(C.byref(p), C.byref(b), stream_h), "ap_render_pass")
        if record:
            e1.record(dev_stream)
            pass_events.append((e0, e1))
        hist = engine.get_scratch_device_array((num_bins,), np.int32, "hist_bins_0")
        cdf = engine.get_scratch_device_array((num_bins,), np.float32, "cdf_lut_0")
        _lib.check(L.ap_histogram_cdf(C.c_void_p(fr.iter.data_ptr()), W, H, wl["max_iter"], num_bins,
                                      C.c_void_p(hist.data_ptr()), C.c_void_p(cdf.data_ptr()),
                                      stream_h), "ap_histogram_cdf")
        b = engine._buffers(fr, lut, cdf=cdf)
        _lib.check(L.ap_colour(C.byref(p), C.byref(b), stream_h), "ap_colour")

    launches_per_step = 4  # render pass, histogram, CDF scan, colour

    for _ in range(args.warmup):
        device_step(False)
    torch.cuda.synchronize()
    iters = nominal_iterations(kmap.cpu().numpy(), wl["max_iter"])

    barrier(world)
    step_ms = []
    with ClockSampler(local_rank) as clocks:
        torch.cuda.synchronize()
        for _ in range(args.steps):
            with torch.cuda.stream(dev_stream):
                flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(dev_stream)
            device_step(True)
            e1.record(dev_stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
    barrier(world)
    total_ms = max_over_ranks(float(np.sum(step_ms)), world)
    pass_ms = float(np.mean([a.elapsed_time(b) for a, b in pass_events]))
    value = iters * args.steps * world / (total_ms * 1e-3) / 1e9

    # End to end through the public entry point with host buffers.
    h_rgb = torch.empty((H, W, 3), dtype=torch.uint8).pin_memory().numpy()
    call = dict(ssaa_factor=wl["factor"], color_scheme_id=wl["scheme"],
                precision_mode=wl["precision_mode"], fractal_type=wl["fractal_type"],
                h_rgb_buf=h_rgb, stream=dev_stream)
    for _ in range(args.warmup):
        engine.render_frame_ssaa(W, H, wl["max_iter"], Decimal(wl["cx"]), Decimal(wl["cy"]),
                                 Decimal(wl["width"]), None, **call)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        engine.render_frame_ssaa(W, H, wl["max_iter"], Decimal(wl["cx"]), Decimal(wl["cy"]),
                                 Decimal(wl["width"]), None, **call)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    barrier(world)
    e2e = iters * args.steps * world / e2e_s / 1e9

    if rank != 0:
        return
    peak64 = fma_peak_tflops(64, stream_h, torch)
    achieved = wl["flops_per_iter"] * iters / (pass_ms * 1e-3) / 1e12
    traffic = load_traffic(wl["name"])
    cpu_value, cpu_sample = cpu_baseline(wl)
    line = {
        "metric": "G iter/s", "value": value, "unit": "G iter/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "ours",
        "config": config_of(wl, args),
        "nominal_iterations_per_frame": iters,
        "e2e": {"value": e2e, "unit": "G iter/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": H * W * 3},
        "roofline": {"bound": wl["bound"], "kernel": "render_pass_kernel", "achieved": achieved,
                     "peak": peak64, "unit": "TFLOP/s", "frac": achieved / peak64 if peak64 else None,
                     "peak_source": "measured dependent-FMA FP64 probe (ap_fma_peak_launch) in this run",
                     "kernel_ms": pass_ms,
                     "traffic": traffic.get("bytes_per_launch") if traffic else None},
        "clocks": clocks.summary(),
        "gpu_launches": launches_per_step * args.steps,
        "cpu_baseline": {"value": cpu_value, "unit": "G iter/s", "cores": os.cpu_count(),
                         "kind": "port", "sample": cpu_sample},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline(wl):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    oracle.set_threads(os.cpu_count() or 1)
    return time_oracle(wl, 3, 1)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local_rank = dist_env()
    wl = WORKLOADS[args.workload]()
    if args.impl == "reference":
        cpu_reference_arm(args, wl, rank, world)
        return
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    try:
        our_arm(args, wl, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
