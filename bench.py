#!/usr/bin/env python
"""Benchmark of the escape-time hot path (G iterations per second).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

Workload (default "cfg3"): 1920x1080 Mandelbrot at width 1e-160 around the
600-digit centre of tests/golden/workloads.json, max_iter 200000, Pauldelbrot
glitch detection with up to 4 rebase passes.  The measured ("chosen") form
uses FP64 deltas and the dc-aware chained-BLA table (bla_form="accurate");
the comparator is the plain FP64-delta form (no BLA) with the same glitch
handling.  A step renders one frame.  The metric is nominal iterations per
second: the sum over pixels of the escape step (max_iter for pixels that never
escape, 0 for cardioid skips), BLA leaps counting the steps they skip.

Rank 0 prints one JSON line:
  value     device-resident throughput of the chosen form: the frame's recorded
            device work (render passes, device BLA builds, rebase passes, device
            copies) replayed with every reference orbit already in HBM; CUDA
            events per step on the launching stream, a 512 MiB write between
            steps (L2 flush), max over ranks;
  e2e       the same metric through engine.render_frame_ssaa with host
            buffers: orbit search (LRU-cached like the reference's), the
            rebase orbits in Decimal, H2D of orbits, D2H of the glitch and
            iteration maps per rebase pass and of the RGB frame;
  plain_fp64_delta, chosen, forms
            per form: G iter/s, and (for the 1e-160 view) the smooth error and
            escape-step agreement against the 700-bit ground truth
            (tests/golden/truth_cfg3.npz) and against the plain form;
  roofline  FP64 pipe of the render passes: executed FP64 operations (from the
            kernels' work counters) / their event-timed duration, against the
            measured dependent-FMA FP64 peak;
  cpu_baseline, clocks, gpu_launches (kernels launched by the library in
            the timed region, from its own counter).
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

# Executed FP64 operations of the perturbation loop (reference-CPU arithmetic, no fused ops):
#   stage-1 step: z = Z + dz (2), |z|^2 (3), Pauldelbrot test (4), BLA radius test (3),
#                 dz' = (2Z + dz) dz + dc (13)                                        -> 25
#   BLA leap:     z, |z|^2 (5), Pauldelbrot test (4), radius test (3), A dz + B dc (14) -> 26
#   stage-2 step: z^2 + c direct (8)
FLOPS_STEP1 = 25.0
FLOPS_LEAP = 26.0
FLOPS_STEP2 = 8.0
FLOPS_DIRECT = 8.0  # FP64 direct Mandelbrot step
# Double-double Burning Ship step, CPU profile (csrc/ap_dd.cuh with the Dekker
# product): two squares (2 x 26), |Z|^2 (1), dd_sub (14), dd_mul of |zx|,|zy| (27),
# doubling (2), dd_add (14), dd_sub (14)                                           -> 124
FLOPS_DD_SHIP = 124.0
# FloatExp perturbation step (FP64 mantissa): the FP64-delta step (25) plus the
# exponent-scaled Z terms and the renormalisation test (10)                          -> 35
FLOPS_STEP1_FEXP = 35.0
# One-pass rebasing (AP_FLAG_REBASE), per step: z = Z + dz (2), |dz|^2 (3, the safe,
# leap and rebase tests), |z|^2 (3, escape and rebase tests), dz' = (2Z + dz) dz + dc (13)
#                                                                                    -> 21
# per leap: z (2), |z|^2 (3), |dz|^2 (3), A dz + B dc (14)                           -> 22
FLOPS_STEP_REBASE = 21.0
FLOPS_LEAP_REBASE = 22.0


# --------------------------------------------------------------- workloads
def _centres():
    with open(os.path.join(ROOT, "tests", "golden", "workloads.json")) as f:
        return json.load(f)


def workload_cfg3():
    cx, cy = _centres()["config3_centre"]
    return dict(name="mandelbrot_perturb_bla_rebase_1920x1080_w1e-160", W=1920, H=1080,
                max_iter=200000, cx=cx, cy=cy, width="1e-160", scheme=0, factor=1, fractal_type=0,
                precision_mode="1e-300 (Perturbation)", bbsa_order=32, bbsa_tol=1e-6,
                glitch_mode="One-Pass Rebasing", arith="ref_cpu", dtype="f64", bla_form="accurate",
                form="FP64 deltas, dc-aware chained BLA (eps 1e-14), one-pass rebasing "
                     "(every pixel restarts its delta when |z| < |dz| or the reference ends; "
                     "no re-render pass)")


def workload_cfg1():
    return dict(name="mandelbrot_fp64_640x360_hist", W=640, H=360, max_iter=1000, cx="-0.65",
                cy="0.0", width="4.0", scheme=11, factor=1, fractal_type=0,
                precision_mode="1e-12 (FP64)", bbsa_order=0, bbsa_tol=0.0,
                glitch_mode="Off (Single-Ref)", arith="ref_cpu", dtype="f64",
                form="FP64 direct iteration, histogram colouring")


def workload_cfg2():
    cx, cy = _centres()["config2_centre"]
    return dict(name="burning_ship_dd_1280x720_w1e-20_ssaa2", W=1280, H=720, max_iter=20000, cx=cx, cy=cy,
                width="1e-20", scheme=0, factor=2, fractal_type=1, precision_mode="1e-24 (DD)",
                bbsa_order=0, bbsa_tol=0.0, glitch_mode="Off (Single-Ref)", arith="ref_cpu", dtype="f64",
                flops_per_iter=FLOPS_DD_SHIP,
                form="double-double direct iteration, 2x adaptive SSAA (coarse, edge mask, edge pass)")


def workload_cfg3b():
    wl = workload_cfg3()
    wl.update(name="mandelbrot_floatexp_bla_pauldelbrot_1920x1080_w1e-1000", width="1e-1000",
              form="FloatExp deltas (FP64 mantissa, int exponent), dc-aware chained BLA (eps 1e-14), "
                   "Pauldelbrot with up to 4 rebase passes")
    return wl


def workload_cfg4():
    tiles = _centres().get("config4_tiles")
    if not tiles:
        raise SystemExit("workloads.json holds no config4_tiles (python tests/golden/make_golden.py config4)")
    return dict(name="batch64_mixed_formulas_perturb_w1e-60_1e-12", kind="batch", tiles=tiles,
                arith="ref_cpu", bla_form="accurate", dtype="f64", W=0, H=0, factor=1,
                max_iter=max(t["max_iter"] for t in tiles), width="1e-60..1e-12",
                bbsa_order=32, glitch_mode="Off (Single-Ref)", precision_mode="1e-300 (Perturbation)",
                scheme=0, fractal_type=-1,
                form="one persistent work-stealing kernel over 64 tiles (FP64 deltas, dc-aware "
                     "chained BLA, Pauldelbrot flags, one reference per tile), CUDA-graph replay, "
                     "autotuned launch shape")


WORKLOADS = {"cfg3": workload_cfg3, "cfg1": workload_cfg1, "cfg2": workload_cfg2, "cfg3b": workload_cfg3b,
             "cfg4": workload_cfg4}
DEFAULT_WORKLOAD = "cfg3"


# ------------------------------------------------------------------ helpers
def dist_env():
    from fractura_b200 import dist
    return dist.env()


class ClockSampler:
    """nvidia-smi clock and throttle-reason sampling during the timed region."""

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
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.perf_counter(), line.strip()))

    def mark(self, start=True):
        if start:
            self.t0 = time.perf_counter()
        else:
            self.t1 = time.perf_counter()

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        t0, t1 = getattr(self, "t0", 0.0), getattr(self, "t1", float("inf"))
        out = self._summary(t0, t1 + 0.05)
        if out["samples"] == 0:
            # a timed region shorter than the sampling interval: the samples nearest to it
            out = self._summary(t0 - 0.1, t1 + 0.1)
            out["window"] = "timed region +-100 ms (shorter than the sampling interval)"
        return out

    def _summary(self, t0, t1):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ts, ln in self.lines:
            if not (t0 <= ts <= t1):
                continue
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


def fma_peak_tflops(precision, torch):
    """Dependent-FMA probe of the FP64/FP32 vector pipe in TFLOP/s (best of 5)."""
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
                                        C.byref(flops), C.c_void_p(st.cuda_stream)),
                   "ap_fma_peak_launch")
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


def nominal_iterations(kmap, max_iter):
    """Escape steps summed; max_iter for never-escaped samples; 0 for cardioid skips."""
    k = np.asarray(kmap)
    return float(k[k >= 0].astype(np.int64).sum() + np.int64(max_iter) * np.count_nonzero(k == -1))


def batch_tiles(wl):
    from fractura_b200 import batch as fb
    return [fb.Tile(cx=Decimal(t["cx"]), cy=Decimal(t["cy"]), width=Decimal(t["width"]), W=t["W"], H=t["H"],
                    max_iter=t["max_iter"], fractal_type=t["fractal_type"], julia_cx=t["julia_cx"],
                    julia_cy=t["julia_cy"], gen_n=t["gen_n"], gen_kr=t["gen_kr"], gen_ki=t["gen_ki"],
                    bla=True, strict_glitch=True) for t in wl["tiles"]]


def config_of(wl, n_gpus):
    if wl.get("kind") == "batch":
        tiles = wl["tiles"]
        kinds = {}
        for t in tiles:
            key = {0: "mandelbrot", 1: "burning_ship", 2: "julia", 3: "ship_julia"}.get(
                t["fractal_type"], f"multibrot{t['gen_n']}")
            kinds[key] = kinds.get(key, 0) + 1
        return {"workload": wl["name"], "tiles": len(tiles), "pixels": sum(t["W"] * t["H"] for t in tiles),
                "formulas": kinds, "max_iter_range": [min(t["max_iter"] for t in tiles),
                                                      max(t["max_iter"] for t in tiles)],
                "width_range": wl["width"], "arith": wl["arith"], "bla_form": wl["bla_form"],
                "form": wl["form"], "l2": "flushed between timed steps (512 MiB write)",
                "parallelism": f"replicas x{n_gpus}" if n_gpus > 1 else "single"}
    return {"workload": wl["name"], "width": wl["W"], "height": wl["H"], "max_iter": wl["max_iter"],
            "view_width": wl["width"], "ssaa": wl["factor"], "bla": wl["bbsa_order"] == 32,
            "glitch_mode": wl["glitch_mode"], "max_rebase_passes": 4, "arith": wl["arith"],
            "form": wl.get("form"), "bla_form": wl.get("bla_form", "reference"),
            "l2": "flushed between timed steps (512 MiB write)",
            "parallelism": f"replicas x{n_gpus}" if n_gpus > 1 else "single"}


def barrier(world):
    from fractura_b200 import dist
    dist.barrier()


def max_over_ranks(x, world):
    from fractura_b200 import dist
    return dist.max_over_ranks(x)


# ----------------------------------------------------------- CPU baseline
def oracle_batch_baseline(wl, budget_s=12.0, start=0):
    """The reference's CPU path, tile by tile (oracle C port, all host cores, chained BLA
    with the reference's table, one reference per tile), on the first tiles of the
    batch until budget_s of CPU time is spent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    from helpers import oracle_pert_frame
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    iters, spent, n = 0.0, 0.0, 0
    order = wl["tiles"][start % len(wl["tiles"]):] + wl["tiles"][:start % len(wl["tiles"])]
    for t in order:
        m = dict(W=t["W"], H=t["H"], factor=1, max_iter=t["max_iter"], cx=t["cx"], cy=t["cy"],
                 width=t["width"], scheme=0, fractal_type=t["fractal_type"], julia_cx=t["julia_cx"],
                 julia_cy=t["julia_cy"], gen_n=t["gen_n"], gen_kr=t["gen_kr"], gen_ki=t["gen_ki"],
                 bbsa_order=32 if t["fractal_type"] in (0, 2, 4) else 0, glitch_mode="Off (Single-Ref)")
        t0 = time.perf_counter()
        fr, _ = oracle_pert_frame(m)
        spent += time.perf_counter() - t0
        iters += nominal_iterations(fr.kmap, t["max_iter"])
        n += 1
        if spent > budget_s:
            break
    return iters / spent / 1e9, cores, (f"{n} of {len(wl['tiles'])} tiles from tile {start % len(wl['tiles'])}, "
                                        f"one pass each incl. host orbits, C port of the reference's "
                                        f"CPU kernels")


def oracle_pert_rows(wl, budget_s, start=0):
    """Rows of a perturbation frame through the oracle (all host cores): the primary
    reference orbit, the reference's BLA table, Pauldelbrot flags, rows start,
    start + 17, ... until budget_s is spent.  Returns (G iter/s, cores, sample)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from fractura_b200 import abi
    from fractura_b200 import high_precision as hp
    from fractura_b200.config import compute_floatexp_scale, decimal_context
    from decimal import localcontext
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    W, H, mi = wl["W"], wl["H"], wl["max_iter"]
    pw = Decimal(wl["width"])
    floatexp = pw < Decimal("1e-300")
    e_scale = compute_floatexp_scale(pw) if floatexp else 0
    with localcontext(decimal_context(pw)):
        ph = pw * (Decimal(H) / Decimal(W))
        two_e = Decimal(2) ** e_scale
        dx = float(pw * two_e / Decimal(W - 1))
        dy = float(ph * two_e / Decimal(H - 1))
    t0 = time.perf_counter()
    bcx, bcy, bu, bv, re, im, rl = hp.find_optimal_reference_orbit(
        Decimal(wl["cx"]), Decimal(wl["cy"]), pw, ph, mi, W, H, is_floatexp=floatexp)
    T = oracle.build_bla(re, im, rl, 0, 1e-6, 16, 3, 0.25, 1.0) if wl["bbsa_order"] == 32 else None
    p = abi.new_params(width=W, height=H, max_iter=mi,
                       tier=abi.AP_TIER_FLOATEXP if floatexp else abi.AP_TIER_PERTURB, e_scale=e_scale,
                       arith=abi.AP_ARITH_REF_CPU, dx_hi=dx, dy_hi=dy, ref_px=(W - 1) * float(bu),
                       ref_py=(H - 1) * float(bv), ref_cx=float(bcx), ref_cy=float(bcy), ref_len=rl,
                       bla_levels=16 if T is not None else 0, strict_glitch=1,
                       flags=abi.AP_FLAG_ESCAPE_GLITCH | abi.AP_FLAG_NAN_GUARD)
    xs = np.arange(W, dtype=np.float64)
    iters, rows = 0.0, 0
    j = start % 17
    while True:
        _, _, k = oracle.pert_grid(p, re[:rl + 1], im[:rl + 1], T, xs, np.array([float(j)]))
        iters += nominal_iterations(k, mi)
        rows += 1
        j += 17
        if j >= H:
            j = (j + 1) % 17
        if time.perf_counter() - t0 > budget_s:
            break
    spent = time.perf_counter() - t0
    return iters / spent / 1e9, cores, (f"{rows} rows of the {W}x{H} frame incl. the host orbit "
                                        f"and BLA table, one reference, C port of the reference's "
                                        f"CPU kernels")


def oracle_baseline(wl, budget_s=12.0, sampled=False, start=0):
    """The reference's per-pixel path restated in C (oracle/) on all host cores, on a
    bounded sample of the workload: the whole frame (direct tiers; perturbation frames
    with their rebase passes unless sampled), rows of it (sampled perturbation frames)
    or whole tiles (batches) until budget_s is spent."""
    if wl.get("kind") == "batch":
        return oracle_batch_baseline(wl, budget_s, start=start)
    direct = wl["precision_mode"].startswith(("1e-12", "1e-24"))
    if sampled and not direct:
        return oracle_pert_rows(wl, budget_s, start=start)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from fractura_b200 import abi
    from fractura_b200 import high_precision as hp
    from fractura_b200.config import decimal_context
    from decimal import localcontext
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    W, H, mi = wl["W"], wl["H"], wl["max_iter"]
    if direct:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from helpers import direct_params, oracle_direct_frame
        m = dict(W=W, H=H, factor=wl["factor"], max_iter=mi, cx=wl["cx"], cy=wl["cy"], width=wl["width"],
                 scheme=wl["scheme"], fractal_type=wl["fractal_type"])
        tier = abi.AP_TIER_FP64 if wl["precision_mode"].startswith("1e-12") else abi.AP_TIER_DD
        if wl["factor"] == 1:
            p = direct_params(m, tier, abi.AP_ARITH_REF_CPU)
            p.flags = abi.AP_FLAG_NO_RGB
            fr = oracle.Frame(W, H)
            t0 = time.perf_counter()
            oracle.render_pass(p, fr)
            t = time.perf_counter() - t0
            return nominal_iterations(fr.kmap, mi) / t / 1e9, cores, f"full {W}x{H} frame, one pass"
        t0 = time.perf_counter()
        fr = oracle_direct_frame(m, tier=tier, arith=abi.AP_ARITH_REF_CPU)
        t = time.perf_counter() - t0
        return (nominal_iterations(fr.kmap, mi) / t / 1e9, cores,
                f"full {W}x{H} frame with its {wl['factor']}x adaptive SSAA passes")
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import oracle_pert_frame
    m = dict(W=W, H=H, factor=wl["factor"], max_iter=mi, cx=wl["cx"], cy=wl["cy"],
             width=wl["width"], scheme=wl["scheme"], fractal_type=wl["fractal_type"],
             julia_cx=0.0, julia_cy=0.0, gen_n=3, gen_kr=0.25, gen_ki=1.0,
             bbsa_order=wl["bbsa_order"], glitch_mode=wl["glitch_mode"])
    t0 = time.perf_counter()
    fr, passes = oracle_pert_frame(m)
    t = time.perf_counter() - t0
    return (nominal_iterations(fr.kmap, mi) / t / 1e9, cores,
            f"full {W}x{H} frame incl. host orbits and {passes} rebase passes, C port of the "
            f"reference's CPU kernels")


def cpu_reference_arm(args, wl, rank, world):
    """--impl reference: the reference's CPU implementation of the path (C port in
    oracle/) on all host cores, rank 0 only."""
    if rank != 0:
        return
    vals = []
    sample = cores = None
    # each step a bounded sample, so that the whole run stays within a few minutes
    budget = min(12.0, max(0.3, 150.0 / max(1, args.steps + args.warmup)))
    for q in range(max(1, args.steps)):
        v, cores, sample = oracle_baseline(wl, budget_s=budget, sampled=True, start=q)
        vals.append(v)
    value = float(np.median(vals))
    line = {"metric": "G iter/s", "value": value, "unit": "G iter/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"], "data": "synthetic",
            "impl": "reference", "config": config_of(wl, args.gpus),
            "cpu_baseline": {"value": value, "unit": "G iter/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "G iter/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------- our arm
def render_call(engine, wl, stream, extra=None, **over):
    kw = dict(ssaa_factor=wl["factor"], color_scheme_id=wl["scheme"],
              precision_mode=wl["precision_mode"], fractal_type=wl["fractal_type"],
              bbsa_tol=wl["bbsa_tol"], bbsa_order=wl["bbsa_order"], glitch_mode=wl["glitch_mode"],
              stream=stream, arith=wl["arith"])
    kw.update(over)
    return engine.render_frame_ssaa(wl["W"], wl["H"], wl["max_iter"], Decimal(wl["cx"]),
                                    Decimal(wl["cy"]), Decimal(wl["width"]), None,
                                    _extra_out=extra, **kw)


def timed_replay(torch, _lib, ops, stream, steps, flush, record_pass=False):
    """Replay recorded device work `steps` times; per-step CUDA events on `stream`,
    L2 flush before each step.  Returns (per-step ms, render-pass event pairs)."""
    step_ms, pass_ev = [], []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        with torch.cuda.stream(stream):
            for fn, args, what in ops:
                if record_pass and what in ("ap_render_pass", "ap_resolve_hist_pass"):
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    _lib.check(fn(*args), what)
                    b.record(stream)
                    pass_ev.append((a, b))
                elif args is None:
                    fn()
                else:
                    _lib.check(fn(*args), what)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    return step_ms, pass_ev


def pass_flops(torch, _lib, abi, ops, stream, H, W, strict, has_bla, direct_flops=FLOPS_DIRECT):
    """Executed FP64 operations of every render pass in one replay, from the work counters."""
    counters = torch.zeros((H, W, 4), dtype=torch.int32, device="cuda")
    f1 = 18.0 + (4.0 if strict else 0.0) + (3.0 if has_bla else 0.0)
    total = 0.0
    launches = 0
    with torch.cuda.stream(stream):
        for fn, args, what in ops:
            if args is None:
                fn()
                continue
            if what in ("ap_render_pass", "ap_resolve_hist_pass"):
                bufs = args[1]._obj
                q = type(bufs).from_buffer_copy(bufs)
                counters.zero_()
                q.counters = C.c_void_p(counters.data_ptr())
                _lib.check(fn(args[0], C.byref(q), args[2]), what)
                c = counters.view(-1, 4).sum(dim=0, dtype=torch.int64).cpu().numpy()
                p = args[0]._obj
                if p.tier in (abi.AP_TIER_FP64, abi.AP_TIER_DD):
                    total += direct_flops * float(c[0])
                elif p.flags & abi.AP_FLAG_REBASE:
                    total += FLOPS_STEP_REBASE * float(c[0]) + FLOPS_LEAP_REBASE * float(c[1])
                elif p.tier == abi.AP_TIER_FLOATEXP:
                    total += (f1 - 25.0 + FLOPS_STEP1_FEXP) * float(c[0]) + FLOPS_LEAP * float(c[1]) + \
                        FLOPS_STEP2 * float(c[2])
                else:
                    total += f1 * float(c[0]) + FLOPS_LEAP * float(c[1]) + FLOPS_STEP2 * float(c[2])
                launches += 1
            else:
                _lib.check(fn(*args), what)
    torch.cuda.synchronize()
    return total, launches


def truth_errors(kmap, s64):
    """Smooth error and escape-step agreement against the 700-bit ground truth of the
    1e-160 view (64 x 64 subsample, tests/golden/truth_cfg3.npz)."""
    path = os.path.join(ROOT, "tests", "golden", "truth_cfg3.npz")
    t = np.load(path)
    truth, rows, cols = t["s"], t["rows"], t["cols"]
    k = kmap[np.ix_(rows, cols)]
    err = np.abs(s64[np.ix_(rows, cols)] - truth)
    return {"p50": float(np.median(err)), "p99": float(np.percentile(err, 99)),
            "p99.9": float(np.percentile(err, 99.9)), "max": float(err.max()),
            "k_identical": float(np.mean(k == np.floor(truth))), "samples": int(err.size)}


class Form:
    """One engine form of the workload: a recorded frame and its replay timings."""

    def __init__(self, name, over, desc):
        self.name, self.over, self.desc = name, over, desc


def record_form(torch, _lib, engine, wl, stream, form, kmap, s64, warm=2):
    from fractura_b200 import high_precision as hp
    hp.clear_reference_orbit_cache()
    for _ in range(warm):
        render_call(engine, wl, stream, (kmap, s64), **form.over)
    torch.cuda.synchronize()
    with _lib.recording() as rec:
        render_call(engine, wl, stream, (kmap, s64), **form.over)
    torch.cuda.synchronize()
    form.ops = rec.ops
    form.kmap = kmap.cpu().numpy()
    form.s64 = s64.cpu().numpy()
    form.iters = nominal_iterations(form.kmap, wl["max_iter"])
    from fractura_b200 import perturbation
    form.stats = dict(perturbation.LAST_FRAME_STATS)
    return form


def summarise_form(form, ms, plain=None, wl=None):
    out = {"form": form.desc, "ms_per_frame": float(np.median(ms)),
           "value": form.iters / (float(np.median(ms)) * 1e-3) / 1e9, "unit": "G iter/s",
           "render_passes": 1 + int(form.stats.get("rebase_passes", 0))}
    if wl is not None and wl["width"] == "1e-160" and wl["W"] == 1920 and wl["H"] == 1080:
        out["error_vs_truth"] = truth_errors(form.kmap, form.s64)
    if plain is not None:
        out["k_identical_vs_plain"] = float(np.mean(form.kmap == plain.kmap))
        out["smooth_diff_vs_plain_p99.9"] = float(np.percentile(np.abs(form.s64 - plain.s64), 99.9))
    return out


def step_flops(fractal_type, gen_n, strict, bla):
    """(stage-1 step, BLA leap, stage-2 step) FP64 operations of coarse_pixel per formula
    (reference-CPU arithmetic, no fused ops): z = Z + dz and |dz|^2 (5), the
    Pauldelbrot test (4 when on), the radius test (3 when BLA is on), then the step:
    z^2 + c 13; Burning Ship 19 (the sign folds); Multibrot 22 per power beyond the
    first plus 10 for K dz + dc.  Stage 2 iterates z directly: 8, 9, 3 + 6 (n - 1) + 10."""
    if fractal_type in (1, 3):
        step, direct = 19.0, 9.0
    elif fractal_type == 4:
        step, direct = 22.0 * (gen_n - 1) + 10.0, 3.0 + 6.0 * (gen_n - 1) + 10.0
    else:
        step, direct = 13.0, 8.0
    return 5.0 + (4.0 if strict else 0.0) + (3.0 if bla else 0.0) + step, FLOPS_LEAP, direct


def batch_flops(torch, _lib, b, cfg):
    """Executed FP64 operations of one batch render, from the kernel's work counters
    (a counter-carrying copy of the descriptors, rendered once outside the timed region)."""
    import ctypes as Cx
    from fractura_b200 import abi
    counters = []
    arr = (abi.ApTileDesc * b.n).from_buffer_copy(b.desc_host)
    for slot, q in enumerate(b.order):
        t = b.tiles[q]
        c = torch.zeros((t.H, t.W, 4), dtype=torch.int32, device="cuda")
        arr[slot].counters = Cx.c_void_p(c.data_ptr())
        counters.append((slot, c))
    keep = b.desc_dev
    b.desc_dev = torch.from_numpy(np.frombuffer(bytes(arr), dtype=np.uint8).copy()).cuda()
    try:
        b.render(cfg)
        torch.cuda.synchronize()
    finally:
        b.desc_dev = keep
    total = 0.0
    for slot, c in counters:
        p = arr[slot].p
        f1, fl, f2 = step_flops(p.fractal_type, p.gen_n, p.strict_glitch > 0, p.bla_levels > 1)
        s = c.view(-1, 4).sum(dim=0, dtype=torch.int64).cpu().numpy()
        total += f1 * float(s[0]) + fl * float(s[1]) + f2 * float(s[2])
    return total


def batch_arm(args, wl, rank, world, local_rank):
    """Config 4: every rank renders the whole 64-tile batch (weak scaling)."""
    import torch
    from fractura_b200 import _lib
    from fractura_b200 import batch as fb
    from fractura_b200 import dist
    from fractura_b200 import high_precision as hp

    torch.cuda.set_device(local_rank)
    stream = torch.cuda.Stream()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    L = _lib.load()
    tiles = batch_tiles(wl)
    hp.clear_reference_orbit_cache()
    b = fb.prepare_batch(tiles, arith=wl["arith"], bla_form=wl["bla_form"], stream=stream)
    cfg = fb.tune(b)
    g = b.capture(cfg)
    for _ in range(args.warmup):
        g.replay()
    torch.cuda.synchronize()
    iters = b.nominal_iterations()

    barrier(world)
    c0 = L.ap_launch_counter()
    step_ms = []
    with ClockSampler(local_rank) as clocks:
        time.sleep(0.5)
        torch.cuda.synchronize()
        clocks.mark(True)
        torch.cuda.nvtx.range_push("timed_region")
        for _ in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            with torch.cuda.stream(stream):
                g.replay()
            e1.record(stream)
            e1.synchronize()
            step_ms.append(e0.elapsed_time(e1))
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        clocks.mark(False)
    # a graph replay launches the batch kernel once; the library's counter does not see it
    launches = (L.ap_launch_counter() - c0) + args.steps
    barrier(world)
    total_ms = max_over_ranks(float(np.sum(step_ms)), world)
    value = dist.whole_job_rate(iters, args.steps, world, total_ms) / 1e9

    # end to end: orbits (host), tables and records (device), the persistent launch and
    # the download of every tile's smooth map, per step
    e2e_steps = max(2, args.steps // 20)
    barrier(world)
    t0 = time.perf_counter()
    h2d = d2h = 0
    for _ in range(e2e_steps):
        hp.clear_reference_orbit_cache()
        bb = fb.prepare_batch(tiles, arith=wl["arith"], bla_form=wl["bla_form"], stream=stream)
        bb.render(cfg)
        maps = [o["iter"].cpu() for o in bb.tiles_out]
        d2h = sum(m.numel() * 4 for m in maps)
        h2d = sum(16 * (p.ref_len + 1) for p in bb.params) + len(bb.desc_dev)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    barrier(world)
    e2e = iters * e2e_steps * world / e2e_s / 1e9
    if rank != 0:
        return
    cpu_value, cores, cpu_sample = oracle_baseline(wl)
    flops = batch_flops(torch, _lib, b, cfg)
    kernel_ms = float(np.median(step_ms))  # the step is the graph's one persistent launch
    peak64 = fma_peak_tflops(64, torch)
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    line = {
        "metric": "G iter/s", "value": value, "unit": "G iter/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"],
        "data": "synthetic", "impl": "ours", "config": config_of(wl, world),
        "nominal_iterations_per_batch": iters,
        "roofline": {"bound": "fp64", "kernel": "batch_kernel (one persistent launch per step)",
                     "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                     "frac": achieved / peak64 if peak64 else None,
                     "peak_source": "measured dependent-FMA FP64 probe (ap_fma_peak_launch), this run",
                     "kernel_ms_per_step": kernel_ms, "traffic": None},
        "e2e": {"value": e2e, "unit": "G iter/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e2e_steps},
        "autotuner": {"chosen": vars(cfg) if hasattr(cfg, "__dict__") else cfg.__repr__(),
                      "candidates_ms": [[round(ms, 4), repr(c)] for ms, c in fb.tuned_timings(b)]},
        "clocks": clocks.summary(),
        "gpu_launches": int(launches),
        "cpu_baseline": {"value": cpu_value, "unit": "G iter/s", "cores": cores, "kind": "port",
                         "sample": cpu_sample},
    }
    print(json.dumps(line), flush=True)


def our_arm(args, wl, rank, world, local_rank):
    import torch
    from fractura_b200 import _lib, abi, engine

    torch.cuda.set_device(local_rank)
    stream = torch.cuda.Stream()
    W, H = wl["W"], wl["H"]
    kmap = torch.empty((H, W), dtype=torch.int32, device="cuda")
    s64 = torch.empty((H, W), dtype=torch.float64, device="cuda")
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    L = _lib.load()
    perturb = wl["bbsa_order"] == 32

    chosen = Form("chosen", dict(bla_form=wl.get("bla_form", "reference")), wl.get("form", ""))
    record_form(torch, _lib, engine, wl, stream, chosen, kmap, s64, warm=args.warmup)

    barrier(world)
    c0 = L.ap_launch_counter()
    with ClockSampler(local_rank) as clocks:
        time.sleep(0.5)  # let the sampler start before the timed region
        torch.cuda.synchronize()
        clocks.mark(True)
        # NVTX range "timed_region": lets a profiler select exactly the timed launches
        torch.cuda.nvtx.range_push("timed_region")
        step_ms, pass_ev = timed_replay(torch, _lib, chosen.ops, stream, args.steps, flush,
                                        record_pass=True)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        clocks.mark(False)
    launches = L.ap_launch_counter() - c0
    barrier(world)
    total_ms = max_over_ranks(float(np.sum(step_ms)), world)
    from fractura_b200 import dist
    value = dist.whole_job_rate(chosen.iters, args.steps, world, total_ms) / 1e9

    # End to end through render_frame_ssaa with a pinned host RGB buffer.
    e2e_steps = max(3, args.steps // 10)
    h_rgb = torch.empty((H, W, 3), dtype=torch.uint8).pin_memory().numpy()
    barrier(world)
    t0 = time.perf_counter()
    from fractura_b200 import high_precision as hp
    for _ in range(e2e_steps):
        hp.clear_reference_orbit_cache()  # every step computes its orbits: a cold frame
        render_call(engine, wl, stream, h_rgb_buf=h_rgb, **chosen.over)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    barrier(world)
    e2e = chosen.iters * e2e_steps * world / e2e_s / 1e9
    from fractura_b200 import perturbation
    h2d = perturbation.LAST_FRAME_STATS["h2d_bytes"] if perturb else 0
    d2h = (perturbation.LAST_FRAME_STATS["d2h_bytes"] if perturb else 0) + H * W * 3

    if rank != 0:
        return
    line_extra = {}
    if perturb:
        n_cmp = max(3, args.steps // 10)
        plain = record_form(torch, _lib, engine, wl, stream,
                            Form("plain", dict(bbsa_order=0, glitch_mode="Pauldelbrot"),
                                 "plain FP64 deltas, no BLA, Pauldelbrot with up to 4 rebase passes "
                                 "(the reference's form)"),
                            kmap, s64)
        p_ms, _ = timed_replay(torch, _lib, plain.ops, stream, n_cmp, flush)
        plain_sum = summarise_form(plain, p_ms, wl=wl)
        chosen_sum = summarise_form(chosen, step_ms, plain=plain, wl=wl)
        forms = {}
        single = dict(glitch_mode="Off (Single-Ref)")
        extra = [
            Form("plain_single_reference", dict(bbsa_order=0, **single),
                 "plain FP64 deltas, one reference, no rebasing"),
            Form("chosen_single_reference", dict(chosen.over, **single),
                 chosen.desc + ", one reference, no rebasing"),
            Form("plain_one_pass", dict(bbsa_order=0), "plain FP64 deltas, no BLA, one-pass rebasing"),
            Form("chosen_pauldelbrot", dict(chosen.over, glitch_mode="Pauldelbrot"),
                 "FP64 deltas, dc-aware chained BLA, Pauldelbrot with up to 4 rebase passes"),
            Form("reference_bla", dict(bla_form="reference", glitch_mode="Pauldelbrot"),
                 "FP64 deltas with the reference's BLA table (tol 1e-6), Pauldelbrot with up to 4 "
                 "rebase passes"),
            Form("fp32_floatexp", dict(chosen.over, delta_form="fp32", glitch_mode="Pauldelbrot"),
                 "FP32 mantissa + int exponent deltas, accurate BLA, Pauldelbrot with up to 4 rebase "
                 "passes"),
        ]
        for f in extra:
            record_form(torch, _lib, engine, wl, stream, f, kmap, s64)
            f_ms, _ = timed_replay(torch, _lib, f.ops, stream, n_cmp, flush)
            forms[f.name] = summarise_form(f, f_ms, plain=plain, wl=wl)
        single_ratio = forms["chosen_single_reference"]["value"] / forms["plain_single_reference"]["value"]
        line_extra = {"plain_fp64_delta": plain_sum, "chosen": chosen_sum,
                      "speedup_vs_plain": value / plain_sum["value"],
                      "speedup_vs_plain_single_reference": single_ratio, "forms": forms}

    strict = "Pauldelbrot" in wl["glitch_mode"] or "Strict" in wl["glitch_mode"]
    flops, n_pass = pass_flops(torch, _lib, abi, chosen.ops, stream, H, W, strict, perturb,
                               wl.get("flops_per_iter", FLOPS_DIRECT))
    pass_ms = float(np.sum([a.elapsed_time(b) for a, b in pass_ev])) / args.steps
    peak64 = fma_peak_tflops(64, torch)
    achieved = flops / (pass_ms * 1e-3) / 1e12 if pass_ms > 0 else None
    traffic = load_traffic(wl["name"])
    cpu_value, cores, cpu_sample = oracle_baseline(wl)
    line = {
        "metric": "G iter/s", "value": value, "unit": "G iter/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"],
        "data": "synthetic", "impl": "ours", "config": config_of(wl, world),
        "nominal_iterations_per_frame": chosen.iters,
        "rebase_passes": int(chosen.stats.get("rebase_passes", 0)),
        "e2e": {"value": e2e, "unit": "G iter/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": e2e_steps},
        **line_extra,
        "roofline": {"bound": "fp64", "kernel": "render passes (perturb_coarse_kernel)" if perturb
                     else "render passes (render_pass_kernel)", "achieved": achieved,
                     "peak": peak64, "unit": "TFLOP/s",
                     "frac": achieved / peak64 if (achieved and peak64) else None,
                     "peak_source": "measured dependent-FMA FP64 probe (ap_fma_peak_launch), this run",
                     "launches_per_step": n_pass, "kernel_ms_per_step": pass_ms,
                     "traffic": traffic.get("bytes_per_launch") if traffic else None},
        "clocks": clocks.summary(),
        "gpu_launches": int(launches),
        "cpu_baseline": {"value": cpu_value, "unit": "G iter/s", "cores": cores, "kind": "port",
                         "sample": cpu_sample},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
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
        if wl.get("kind") == "batch":
            batch_arm(args, wl, rank, world, local_rank)
        else:
            our_arm(args, wl, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
