#!/usr/bin/env python
"""Benchmark of the escape-time hot path (G iterations per second).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]
                    [--configs auto|none]

Headline workload (default "cfg3"): 1920x1080 Mandelbrot at width 1e-160 around the
600-digit centre of tests/golden/workloads.json, max_iter 200000.  The measured form
uses FP64 deltas, the dc-aware chained-BLA table (bla_form="accurate") and one-pass
rebasing (glitch_mode "One-Pass Rebasing": every pixel restarts its delta when
|z| < |dz| or the reference ends, in the same pass).  A step renders one frame.  The
metric is nominal iterations per second: the sum over pixels of the escape step
(max_iter for pixels that never escape, 0 for cardioid skips), BLA leaps counting the
steps they skip.

Rank 0 prints one JSON line:
  value     device-resident throughput: the frame's recorded device work (render
            passes, device BLA build, device copies) replayed with the reference orbit
            already in HBM; CUDA events per step on the launching stream, a 512 MiB
            write between steps (L2 flush), max over ranks;
  e2e       the same metric through engine.render_frame_ssaa with host buffers: cold
            orbit search on the host (cache cleared every step), H2D of the orbit,
            D2H of the RGB frame (and of the glitch maps where rebase passes run);
  plain_fp64_delta, chosen, forms
            per form: G iter/s and the smooth error / escape-step agreement against the
            700-bit ground truth (tests/golden/truth_cfg3.npz); the plain form is the
            reference's (FP64 deltas, no BLA, Pauldelbrot with up to 4 rebase passes);
  roofline  FP64 pipe of the render passes: executed FP64 operations (from the kernels'
            work counters) / their event-timed duration, against the dependent-FMA FP64
            peak measured in the same run;
  cpu_baseline  the reference's CPU path restated in C (oracle/), all host cores, full
            frames in the reference's own form (Pauldelbrot, its BLA table, orbits from
            oracle/ref_orbit.py);
  configs   with --configs auto (default for cfg3 on one GPU): one record per other
            config (cfg1, cfg2, cfg3b, cfg4, cfg5) with its own value, roofline,
            cpu_baseline and e2e;
  clocks, gpu_launches (kernels launched by the library in the timed region).
Multi-GPU: one process per GPU, every rank renders its own frame (weak scaling, no
collective on the data path).

--impl reference: the reference's CPU implementation of the path (the C port in
oracle/, orbits in Decimal through oracle/ref_orbit.py; no engine code) on all host
cores, full frames, rank 0 only.
"""
import argparse
import ctypes as C
import json
import math
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
# Derivatives of the smooth value (csrc/ap_adjoint.cu), per iteration of a pixel's orbit:
#   forward:  |z|^2 (3) + f(z) and f'(z): z^2 + c (8) and 2z (2)                       -> 13
#             Multibrot n: z^(n-1) (6 (n-1)), z^n and P z (12), sums (4), f' (4), |z|^2 (3)
#   adjoint:  the step twice more (the segment's sub-checkpoint replay and the
#             sub-segment's replay into shared memory: 2 x 10; Multibrot 2 x (6 (n-1) + 20)),
#             the reverse step's f' (2; Multibrot 6 (n-1) + 4), G conj(f') (6), parameter
#             sums (2; Multibrot 10)                                                 -> 30
FLOPS_FWD_QUAD = 13.0
FLOPS_ADJ_QUAD = 30.0


def flops_fwd_multi(n):
    return 6.0 * (n - 1) + 23.0


def flops_adj_multi(n):
    return 18.0 * (n - 1) + 60.0


L2_FLUSH = "flushed between timed steps (512 MiB write)"


# --------------------------------------------------------------- workloads
def _centres():
    with open(os.path.join(ROOT, "tests", "golden", "workloads.json")) as f:
        return json.load(f)


def workload_cfg3():
    cx, cy = _centres()["config3_centre"]
    return dict(name="mandelbrot_perturb_1920x1080_w1e-160_maxiter200000", W=1920, H=1080,
                max_iter=200000, cx=cx, cy=cy, width="1e-160", scheme=0, factor=1, fractal_type=0,
                precision_mode="1e-300 (Perturbation)", bbsa_order=32, bbsa_tol=1e-6,
                glitch_mode="One-Pass Rebasing", arith="fast", dtype="f64", bla_form="accurate",
                form="FP64 deltas, dc-aware chained BLA (eps 1e-14), one-pass rebasing "
                     "(every pixel restarts its delta when |z| < |dz| or the reference ends; "
                     "no re-render pass), fused-multiply-add step (arith 'fast')",
                ref_form="FP64 deltas, the reference's chained BLA (tol 1e-6), Pauldelbrot with up to "
                         "4 rebase passes")


def workload_cfg1():
    return dict(name="mandelbrot_fp64_640x360_w4_maxiter1000_hist", W=640, H=360, max_iter=1000, cx="-0.65",
                cy="0.0", width="4.0", scheme=11, factor=1, fractal_type=0,
                precision_mode="1e-12 (FP64)", bbsa_order=0, bbsa_tol=0.0,
                glitch_mode="Off (Single-Ref)", arith="ref_cpu", dtype="f64",
                form="FP64 direct iteration, histogram colouring (65536-bin CDF)")


def workload_cfg2():
    cx, cy = _centres()["config2_centre"]
    return dict(name="burning_ship_dd_1280x720_w1e-20_maxiter20000_ssaa2", W=1280, H=720, max_iter=20000,
                cx=cx, cy=cy, width="1e-20", scheme=0, factor=2, fractal_type=1, precision_mode="1e-24 (DD)",
                bbsa_order=0, bbsa_tol=0.0, glitch_mode="Off (Single-Ref)", arith="ref_cpu", dtype="f64",
                flops_per_iter=FLOPS_DD_SHIP,
                form="double-double direct iteration, 2x adaptive SSAA (coarse, edge mask, edge pass)")


def workload_cfg3b():
    wl = workload_cfg3()
    wl.update(name="mandelbrot_floatexp_1920x1080_w1e-1000_maxiter200000", width="1e-1000",
              glitch_mode="Pauldelbrot", arith="ref_cuda",
              form="FloatExp deltas (FP64 mantissa, int exponent), dc-aware chained BLA (eps 1e-14), "
                   "Pauldelbrot with up to 4 rebase passes")
    return wl


def workload_cfg4():
    tiles = _centres().get("config4_tiles")
    if not tiles:
        raise SystemExit("workloads.json holds no config4_tiles (python tests/golden/make_golden.py config4)")
    return dict(name="batch64_mixed_formulas_w1e-60_1e-12", kind="batch", tiles=tiles,
                arith="fast", bla_form="accurate", dtype="f64", W=0, H=0, factor=1,
                max_iter=max(t["max_iter"] for t in tiles), width="1e-60..1e-12",
                bbsa_order=32, glitch_mode="One-Pass Rebasing", precision_mode="1e-300 (Perturbation)",
                scheme=0, fractal_type=-1,
                form="one persistent work-stealing kernel over 64 tiles, the unfinished pixels of "
                     "each block compacted between quanta (FP64 deltas, dc-aware chained BLA, one "
                     "reference per tile: one-pass rebasing with the fused step for the Mandelbrot, "
                     "Burning Ship and Multibrot tiles, Pauldelbrot flags in the CUDA-source "
                     "profile for the Julia tiles), CUDA-graph replay, autotuned launch shape")


def workload_cfg5():
    return dict(name="grad_julia_multibrot3_512x512_w3_maxiter2000", kind="adjoint", W=512, H=512,
                max_iter=2000, width="3.0", dtype="f64", arith="ref_cuda", seed=20250,
                cases=[dict(fractal_type=2, gen_n=2, theta=[0.0, 0.0, math.log(3.0), -0.8, 0.156]),
                       dict(fractal_type=4, gen_n=3, theta=[0.0, 0.0, math.log(3.0), 0.1, 0.2])],
                form="FP64 forward with orbit checkpoints every 1024 steps, then the adjoint sweep "
                     "(segments recomputed from checkpoints) for d loss / d(cx, cy, ln w, Re P, Im P); "
                     "Julia j=-0.8+0.156i and Multibrot n=3, k=0.1+0.2i; loss = mean squared "
                     "difference to a target at theta + N(0, 1e-3)")


WORKLOADS = {"cfg3": workload_cfg3, "cfg1": workload_cfg1, "cfg2": workload_cfg2, "cfg3b": workload_cfg3b,
             "cfg4": workload_cfg4, "cfg5": workload_cfg5}
DEFAULT_WORKLOAD = "cfg3"
SUB_RECORDS = ("cfg1", "cfg2", "cfg3b", "cfg4", "cfg5")


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


_PEAKS = {}


def fma_peak_tflops(precision, torch):
    """Dependent-FMA probe of the FP64/FP32 vector pipe in TFLOP/s (best of 5; once per run)."""
    if precision in _PEAKS:
        return _PEAKS[precision]
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
    _PEAKS[precision] = best
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
    rebase = "One-Pass" in wl.get("glitch_mode", "")
    return [fb.Tile(cx=Decimal(t["cx"]), cy=Decimal(t["cy"]), width=Decimal(t["width"]), W=t["W"], H=t["H"],
                    max_iter=t["max_iter"], fractal_type=t["fractal_type"], julia_cx=t["julia_cx"],
                    julia_cy=t["julia_cy"], gen_n=t["gen_n"], gen_kr=t["gen_kr"], gen_ki=t["gen_ki"],
                    bla=True, strict_glitch=True, rebase=rebase and t["fractal_type"] in (0, 1, 4))
            for t in wl["tiles"]]


def batch_fp32_form(torch, fb, hp, wl, b64, cfg, stream, flush, steps):
    """Config 4 in the FP32-mantissa FloatExp form: the same tiles (one-pass rebasing where
    the FP64 batch rebases) with delta_form="fp32", rendered in one persistent launch, and
    its agreement with the FP64 batch b64: identical escape steps and smooth differences
    where both escape at the same step, per formula."""
    import dataclasses
    hp.clear_reference_orbit_cache()
    tiles = [dataclasses.replace(t, delta_form="fp32") for t in batch_tiles(wl)]
    b = fb.prepare_batch(tiles, arith="ref_cuda", bla_form=wl["bla_form"], stream=stream)
    b.render(cfg)
    torch.cuda.synchronize()
    ms = timed_loop(torch, stream, flush, max(3, steps // 5), lambda: b.render(cfg))
    iters = b.nominal_iterations()
    per, same_k, pixels, diffs = {}, 0, 0, []
    for t, o32, o64 in zip(tiles, b.tiles_out, b64.tiles_out):
        k32, k64 = o32["kmap"].cpu().numpy(), o64["kmap"].cpu().numpy()
        s32, s64 = o32["iter"].cpu().numpy(), o64["iter"].cpu().numpy()
        key = {0: "mandelbrot", 1: "burning_ship", 2: "julia", 3: "ship_julia"}.get(
            t.fractal_type, f"multibrot{t.gen_n}")
        eq = k32 == k64
        both = eq & (k64 >= 0)
        d = np.abs(s32[both].astype(np.float64) - s64[both].astype(np.float64))
        diffs.append(d)
        acc = per.setdefault(key, [0, 0])
        acc[0] += int(eq.sum())
        acc[1] += eq.size
        same_k += int(eq.sum())
        pixels += eq.size
    d = np.concatenate(diffs) if diffs else np.zeros(1)
    return {
        "form": "the same tiles with FP32-mantissa FloatExp deltas (24-bit mantissas, int exponents; FP64 "
                "escape, rebase and sign tests where a float screen says they can fire), one persistent launch",
        "value": iters / (float(np.median(ms)) * 1e-3) / 1e9, "unit": "G iter/s",
        "ms_per_batch": float(np.median(ms)),
        "vs_fp64_batch": {"identical_k": same_k / max(1, pixels),
                          "identical_k_by_formula": {k: v[0] / max(1, v[1]) for k, v in sorted(per.items())},
                          "smooth_p99_where_k_equal": float(np.percentile(d, 99)) if d.size else 0.0}}


def config_of(wl, n_gpus):
    """The workload (what is rendered), the same for both arms; the method is "form"."""
    par = f"replicas x{n_gpus}" if n_gpus > 1 else "single"
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
                "width_range": wl["width"], "l2": L2_FLUSH, "parallelism": par}
    if wl.get("kind") == "adjoint":
        return {"workload": wl["name"], "width": wl["W"], "height": wl["H"], "max_iter": wl["max_iter"],
                "view_width": wl["width"], "formulas": ["julia", "multibrot3"], "l2": L2_FLUSH,
                "parallelism": par}
    return {"workload": wl["name"], "width": wl["W"], "height": wl["H"], "max_iter": wl["max_iter"],
            "view_width": wl["width"], "ssaa": wl["factor"], "colour_scheme": wl["scheme"],
            "fractal_type": wl["fractal_type"], "l2": L2_FLUSH, "parallelism": par}


def barrier(world):
    from fractura_b200 import dist
    dist.barrier()


def max_over_ranks(x, world):
    from fractura_b200 import dist
    return dist.max_over_ranks(x)


def timed_loop(torch, stream, flush, steps, body):
    """CUDA-event time of `body()` per step on `stream`, an L2 flush before each step."""
    ms = []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        with torch.cuda.stream(stream):
            body()
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return ms


# ----------------------------------------------------------- CPU baseline
def _oracle_modules():
    for d in ("oracle", "tests"):
        p = os.path.join(ROOT, d)
        if p not in sys.path:
            sys.path.insert(0, p)
    import frames
    import oracle
    return oracle, frames


def reference_view(wl):
    """The workload as a view dict of oracle/frames.py, in the reference's own form."""
    return dict(W=wl["W"], H=wl["H"], factor=wl["factor"], max_iter=wl["max_iter"], cx=wl["cx"], cy=wl["cy"],
                width=wl["width"], scheme=wl["scheme"], fractal_type=wl["fractal_type"], julia_cx=0.0,
                julia_cy=0.0, gen_n=3, gen_kr=0.25, gen_ki=1.0, bbsa_order=wl["bbsa_order"],
                bbsa_tol=wl.get("bbsa_tol", 1e-6), glitch_mode="Pauldelbrot" if wl["bbsa_order"] == 32
                else wl["glitch_mode"])


def cpu_reference_frames(wl, budget_s, max_frames, min_frames=1):
    """The reference's CPU path (oracle C port + Decimal orbit search, no engine code) on
    all host cores: full frames until budget_s is spent.  Returns (per-frame G iter/s,
    per-frame seconds, cores, sample description)."""
    oracle, frames = _oracle_modules()
    cores = os.cpu_count() or 1
    oracle.set_threads(cores)
    kind = wl.get("kind")
    if kind == "batch":
        return cpu_reference_tiles(wl, budget_s)
    if kind == "adjoint":
        return cpu_adjoint_baseline(wl, budget_s)
    direct = wl["precision_mode"].startswith(("1e-12", "1e-24"))
    rates, secs, passes = [], [], 0
    while len(rates) < max_frames and (sum(secs) < budget_s or len(rates) < min_frames):
        t0 = time.perf_counter()
        if direct:
            from helpers import oracle_direct_frame
            from fractura_b200 import abi
            m = dict(W=wl["W"], H=wl["H"], factor=wl["factor"], max_iter=wl["max_iter"], cx=wl["cx"],
                     cy=wl["cy"], width=wl["width"], scheme=wl["scheme"], fractal_type=wl["fractal_type"])
            tier = abi.AP_TIER_FP64 if wl["precision_mode"].startswith("1e-12") else abi.AP_TIER_DD
            fr = oracle_direct_frame(m, tier=tier, arith=abi.AP_ARITH_REF_CPU)
        else:
            fr, passes = frames.pert_frame(reference_view(wl))
        dt = time.perf_counter() - t0
        secs.append(dt)
        rates.append(nominal_iterations(fr.kmap, wl["max_iter"]) / dt / 1e9)
    if direct:
        sample = (f"{len(rates)} full {wl['W']}x{wl['H']} frame(s) with every pass of the reference's "
                  f"path (C port of its CPU kernels)")
    else:
        sample = (f"{len(rates)} full {wl['W']}x{wl['H']} frame(s) in the reference's form: Decimal "
                  f"orbit search (centre + 16-candidate probe, oracle/ref_orbit.py), its BLA table "
                  f"(tol 1e-6), Pauldelbrot with {passes} rebase passes; C port of its CPU kernels")
    return rates, secs, cores, sample


def cpu_reference_tiles(wl, budget_s):
    """Config 4 tile by tile in the reference's form (one reference per tile, its BLA table
    for Mandelbrot/Julia/Multibrot), until budget_s is spent."""
    _, frames = _oracle_modules()
    iters, spent, n = 0.0, 0.0, 0
    for t in wl["tiles"]:
        m = dict(W=t["W"], H=t["H"], factor=1, max_iter=t["max_iter"], cx=t["cx"], cy=t["cy"],
                 width=t["width"], scheme=0, fractal_type=t["fractal_type"], julia_cx=t["julia_cx"],
                 julia_cy=t["julia_cy"], gen_n=t["gen_n"], gen_kr=t["gen_kr"], gen_ki=t["gen_ki"],
                 bbsa_order=32 if t["fractal_type"] in (0, 2, 4) else 0, bbsa_tol=1e-6,
                 glitch_mode="Off (Single-Ref)")
        t0 = time.perf_counter()
        fr, _ = frames.pert_frame(m)
        spent += time.perf_counter() - t0
        iters += nominal_iterations(fr.kmap, t["max_iter"])
        n += 1
        if spent > budget_s:
            break
    return [iters / spent / 1e9], [spent], os.cpu_count() or 1, (
        f"{n} of {len(wl['tiles'])} tiles, one frame each incl. the Decimal orbit search "
        f"(oracle/ref_orbit.py); C port of the reference's CPU kernels")


def cpu_adjoint_baseline(wl, budget_s):
    """Config 5 on the CPU: the oracle's FP64 forward samples (the reference's
    cpu_compute_fp64_sample restated) of both formulas.  The reference has no
    derivative; a central-difference gradient of the 5 parameters takes 10 such forward
    frames, so the CPU gradient rate is a tenth of the forward rate reported here."""
    oracle, _ = _oracle_modules()
    from fractura_b200 import abi
    W, H, mi = wl["W"], wl["H"], wl["max_iter"]
    iters, spent = 0.0, 0.0
    while True:
        for case in wl["cases"]:
            th = case["theta"]
            w = math.exp(th[2])
            h = w * H / W
            xs = (th[0] - 0.5 * w) + np.arange(W) * (w / (W - 1))
            ys = (th[1] + 0.5 * h) - np.arange(H) * (h / (H - 1))
            p = abi.new_params(width=W, height=H, max_iter=mi, fractal_type=case["fractal_type"],
                               gen_n=case["gen_n"], gen_kr=th[3], gen_ki=th[4], tier=abi.AP_TIER_FP64,
                               arith=abi.AP_ARITH_REF_CPU, julia_cx_hi=th[3], julia_cy_hi=th[4])
            t0 = time.perf_counter()
            _, _, k = oracle.fp64_grid(p, xs, ys)
            spent += time.perf_counter() - t0
            iters += nominal_iterations(k, mi)
        if spent > budget_s:
            break
    return [iters / spent / 1e9], [spent], os.cpu_count() or 1, (
        "FP64 forward frames of both formulas through the oracle (C port of "
        "cpu_compute_fp64_sample), all host cores; forward only -- a central-difference "
        "gradient costs 10 such frames per parameter set")


def cpu_baseline_record(wl, budget_s, max_frames=1):
    rates, _, cores, sample = cpu_reference_frames(wl, budget_s, max_frames)
    return {"value": float(np.median(rates)), "unit": "G iter/s", "cores": cores, "kind": "port",
            "sample": sample}


def cpu_reference_arm(args, wl, rank, world):
    """--impl reference: the reference's CPU implementation of the path, rank 0 only.
    Each step is one full frame in the reference's form; the number of timed frames is
    bounded (150 s) so that the run ends within a few minutes."""
    if rank != 0:
        return
    cpu_reference_frames(wl, 0.0, 1)  # one warm-up frame (page-in, thread start)
    rates, secs, cores, sample = cpu_reference_frames(wl, 150.0, max(1, args.steps))
    value = float(np.median(rates))
    line = {"metric": "G iter/s", "value": value, "unit": "G iter/s", "n_gpus": args.gpus,
            "steps": len(rates), "steps_requested": args.steps, "warmup": 1,
            "ms_per_step": float(np.median(secs)) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"], "data": "synthetic",
            "impl": "reference", "config": config_of(wl, args.gpus),
            "form": wl.get("ref_form", wl.get("form")),
            "cpu_baseline": {"value": value, "unit": "G iter/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "G iter/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# -------------------------------------------------------------- frame arm
def render_call(engine, wl, stream, extra=None, **over):
    kw = dict(ssaa_factor=wl["factor"], color_scheme_id=wl["scheme"],
              precision_mode=wl["precision_mode"], fractal_type=wl["fractal_type"],
              bbsa_tol=wl["bbsa_tol"], bbsa_order=wl["bbsa_order"], glitch_mode=wl["glitch_mode"],
              stream=stream, arith=wl["arith"], bla_form=wl.get("bla_form"))
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
    work = np.zeros(4, np.int64)  # steps, leaps, stage-2 steps, rebases (one-pass)
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
                work += c.astype(np.int64)
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
    return total, launches, work


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
            "k_identical": float(np.mean(k == np.floor(truth))), "samples": int(err.size),
            "meets_bound": bool(np.percentile(err, 99) <= 1e-4 and np.mean(k == np.floor(truth)) >= 0.999)}


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


def frame_arm(args, wl, rank, world, local_rank, steps, headline):
    """A frame workload: recorded device work replayed `steps` times (value), the same
    frame through render_frame_ssaa with host buffers (e2e), comparator forms (perturbation
    views) and the roofline of the render passes."""
    import torch
    from fractura_b200 import _lib, abi, dist, engine, perturbation
    from fractura_b200 import high_precision as hp

    stream = torch.cuda.Stream()
    W, H = wl["W"], wl["H"]
    kmap = torch.empty((H, W), dtype=torch.int32, device="cuda")
    s64 = torch.empty((H, W), dtype=torch.float64, device="cuda")
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    L = _lib.load()
    perturb = not wl["precision_mode"].startswith(("1e-12", "1e-24"))

    chosen = Form("chosen", {}, wl.get("form", ""))
    record_form(torch, _lib, engine, wl, stream, chosen, kmap, s64, warm=args.warmup)

    barrier(world)
    c0 = L.ap_launch_counter()
    with ClockSampler(local_rank) as clocks:
        time.sleep(0.3)
        torch.cuda.synchronize()
        clocks.mark(True)
        torch.cuda.nvtx.range_push("timed_region")
        step_ms, pass_ev = timed_replay(torch, _lib, chosen.ops, stream, steps, flush, record_pass=True)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        clocks.mark(False)
    launches = L.ap_launch_counter() - c0
    barrier(world)
    total_ms = max_over_ranks(float(np.sum(step_ms)), world)
    value = dist.whole_job_rate(chosen.iters, steps, world, total_ms) / 1e9

    # End to end through render_frame_ssaa with a pinned host RGB buffer, cold orbit search.
    e2e_steps = max(3, steps // 10)
    h_rgb = torch.empty((H, W, 3), dtype=torch.uint8).pin_memory().numpy()
    render_call(engine, wl, stream, h_rgb_buf=h_rgb)  # warm-up: the host-buffer path's first call
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        hp.clear_reference_orbit_cache()
        render_call(engine, wl, stream, h_rgb_buf=h_rgb)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    barrier(world)
    e2e = chosen.iters * e2e_steps * world / e2e_s / 1e9
    h2d = perturbation.LAST_FRAME_STATS["h2d_bytes"] if perturb else 0
    d2h = (perturbation.LAST_FRAME_STATS["d2h_bytes"] if perturb else 0) + H * W * 3

    if rank != 0:
        return None
    line = {"metric": "G iter/s", "value": value, "unit": "G iter/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": total_ms / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"], "data": "synthetic",
            "impl": "ours", "config": config_of(wl, world), "form": wl.get("form"),
            "arith": wl["arith"], "bla_form": wl.get("bla_form", "reference"),
            "nominal_iterations_per_frame": chosen.iters,
            "rebase_passes": int(chosen.stats.get("rebase_passes", 0)),
            "e2e": {"value": e2e, "unit": "G iter/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                    "path": "engine.render_frame_ssaa, pinned host RGB buffer, orbit cache cleared per step"}}
    if perturb and wl["width"] == "1e-160" and headline:
        n_cmp = max(3, steps // 10)
        plain = record_form(torch, _lib, engine, wl, stream,
                            Form("plain", dict(bbsa_order=0, glitch_mode="Pauldelbrot", bla_form=None,
                                               arith="ref_cuda"),
                                 "plain FP64 deltas, no BLA, Pauldelbrot with up to 4 rebase passes "
                                 "(the reference's CUDA form)"),
                            kmap, s64)
        p_ms, _ = timed_replay(torch, _lib, plain.ops, stream, n_cmp, flush)
        plain_sum = summarise_form(plain, p_ms, wl=wl)
        chosen_sum = summarise_form(chosen, step_ms, plain=plain, wl=wl)
        forms = {}
        single = dict(glitch_mode="Off (Single-Ref)")
        cuda = dict(arith="ref_cuda")
        extra = [
            Form("chosen_ref_cuda", dict(cuda), "the chosen form in the CUDA-source arithmetic profile"),
            Form("chosen_ref_cpu", dict(arith="ref_cpu"), "the chosen form in the CPU-kernel arithmetic "
                                                          "profile (no fused multiply-adds)"),
            Form("plain_single_reference", dict(bbsa_order=0, bla_form=None, **single, **cuda),
                 "plain FP64 deltas, one reference, no rebasing"),
            Form("chosen_single_reference", dict(single, **cuda),
                 "FP64 deltas, dc-aware chained BLA, one reference, no rebasing"),
            Form("plain_one_pass", dict(bbsa_order=0, bla_form=None),
                 "plain FP64 deltas, no BLA, one-pass rebasing"),
            Form("chosen_pauldelbrot", dict(glitch_mode="Pauldelbrot", **cuda),
                 "FP64 deltas, dc-aware chained BLA, Pauldelbrot with up to 4 rebase passes"),
            Form("reference_bla", dict(bla_form="reference", glitch_mode="Pauldelbrot", **cuda),
                 "FP64 deltas with the reference's BLA table (tol 1e-6), Pauldelbrot with up to 4 "
                 "rebase passes"),
            Form("fp32_floatexp", dict(delta_form="fp32", glitch_mode="Pauldelbrot", **cuda),
                 "FP32 mantissa + int exponent deltas, dc-aware BLA, Pauldelbrot with up to 4 rebase "
                 "passes"),
            Form("fp32_floatexp_one_pass", dict(delta_form="fp32", **cuda),
                 "FP32 mantissa + int exponent deltas, dc-aware BLA, one-pass rebasing"),
        ]
        for f in extra:
            record_form(torch, _lib, engine, wl, stream, f, kmap, s64)
            f_ms, _ = timed_replay(torch, _lib, f.ops, stream, n_cmp, flush)
            forms[f.name] = summarise_form(f, f_ms, plain=plain, wl=wl)
        line.update({"plain_fp64_delta": plain_sum, "chosen": chosen_sum,
                     "speedup_vs_plain": value / plain_sum["value"],
                     "speedup_vs_plain_single_reference":
                         forms["chosen_single_reference"]["value"] / forms["plain_single_reference"]["value"],
                     "forms": forms})
    elif perturb and wl["width"] == "1e-1000":
        # the FP32-mantissa form against the FP64-mantissa FloatExp form of the same view
        n_cmp = max(3, steps // 10)
        line["forms"] = {}
        for form in (Form("fp32_floatexp", dict(delta_form="fp32"),
                          "FP32 mantissa + int exponent deltas, dc-aware BLA, Pauldelbrot"),
                     Form("fp32_floatexp_one_pass", dict(delta_form="fp32", glitch_mode="One-Pass Rebasing"),
                          "FP32 mantissa + int exponent deltas, dc-aware BLA, one-pass rebasing")):
            f = record_form(torch, _lib, engine, wl, stream, form, kmap, s64)
            f_ms, _ = timed_replay(torch, _lib, f.ops, stream, n_cmp, flush)
            s = summarise_form(f, f_ms)
            s["k_identical_vs_fp64_floatexp"] = float(np.mean(f.kmap == chosen.kmap))
            d = np.abs(f.s64 - chosen.s64)
            s["smooth_diff_vs_fp64_floatexp"] = {"p50": float(np.median(d)), "p99": float(np.percentile(d, 99)),
                                                 "max": float(d.max())}
            line["forms"][form.name] = s

    strict = "Pauldelbrot" in wl["glitch_mode"] or "Strict" in wl["glitch_mode"]
    flops, n_pass, work = pass_flops(torch, _lib, abi, chosen.ops, stream, H, W, strict,
                                     wl["bbsa_order"] == 32, wl.get("flops_per_iter", FLOPS_DIRECT))
    if perturb:
        # what the render passes executed per frame (work counters): steps taken one at a
        # time, BLA leaps, direct stage-2 steps, one-pass restarts
        line["work_per_frame"] = {"steps": int(work[0]), "leaps": int(work[1]), "stage2_steps": int(work[2]),
                                  "rebases": int(work[3]),
                                  "nominal_iterations": line.get("nominal_iterations_per_frame")}
    pass_ms = float(np.sum([a.elapsed_time(b) for a, b in pass_ev])) / steps
    peak64 = fma_peak_tflops(64, torch)
    achieved = flops / (pass_ms * 1e-3) / 1e12 if pass_ms > 0 else None
    traffic = load_traffic(wl["name"])
    kern = "perturb_coarse_kernel" if perturb else "render_pass_kernel"
    line["roofline"] = {"bound": "fp64", "kernel": f"render passes ({kern})", "achieved": achieved,
                        "peak": peak64, "unit": "TFLOP/s",
                        "frac": achieved / peak64 if (achieved and peak64) else None,
                        "peak_source": "measured dependent-FMA FP64 probe (ap_fma_peak_launch), this run "
                                       "(MEASURED_PEAKS.json holds no FP64 figure)",
                        "launches_per_step": n_pass, "kernel_ms_per_step": pass_ms,
                        "kernel_share_of_step": pass_ms / float(np.median(step_ms)),
                        "traffic": traffic.get("bytes_per_launch") if traffic else None}
    line["clocks"] = clocks.summary()
    line["gpu_launches"] = int(launches)
    return line


# -------------------------------------------------------------- batch arm
def step_flops(fractal_type, gen_n, strict, bla, rebase=False):
    """(stage-1 step, BLA leap, stage-2 step) FP64 operations of coarse_pixel per formula
    (reference-CPU arithmetic, no fused ops): z = Z + dz and |dz|^2 (5), the
    Pauldelbrot test (4 when on), the radius test (3 when BLA is on), then the step:
    z^2 + c 13; Burning Ship 19 (the sign folds); Multibrot 22 per power beyond the
    first plus 10 for K dz + dc.  Stage 2 iterates z directly: 8, 9, 3 + 6 (n - 1) + 10.
    One-pass rebasing (rebase_advance): z and |dz|^2 (5), |z|^2 (3), the step; leaps 22;
    no stage 2."""
    if fractal_type in (1, 3):
        step, direct = 19.0, 9.0
    elif fractal_type == 4:
        step, direct = 22.0 * (gen_n - 1) + 10.0, 3.0 + 6.0 * (gen_n - 1) + 10.0
    else:
        step, direct = 13.0, 8.0
    if rebase:
        return 8.0 + step, FLOPS_LEAP_REBASE, 0.0
    return 5.0 + (4.0 if strict else 0.0) + (3.0 if bla else 0.0) + step, FLOPS_LEAP, direct


def batch_flops(torch, _lib, b, cfg):
    """Executed FP64 operations of one batch render, from the kernel's work counters
    (a counter-carrying copy of the descriptors, rendered once outside the timed region)."""
    from fractura_b200 import abi
    counters = []
    arr = (abi.ApTileDesc * b.n).from_buffer_copy(b.desc_host)
    for slot, q in enumerate(b.order):
        t = b.tiles[q]
        c = torch.zeros((t.H, t.W, 4), dtype=torch.int32, device="cuda")
        arr[slot].counters = C.c_void_p(c.data_ptr())
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
        f1, fl, f2 = step_flops(p.fractal_type, p.gen_n, p.strict_glitch > 0, p.bla_levels > 1,
                                bool(p.flags & abi.AP_FLAG_REBASE))
        s = c.view(-1, 4).sum(dim=0, dtype=torch.int64).cpu().numpy()
        total += f1 * float(s[0]) + fl * float(s[1]) + f2 * float(s[2])
    return total


def batch_arm(args, wl, rank, world, local_rank, steps, headline):
    """Config 4: every rank renders the whole 64-tile batch (weak scaling)."""
    import torch
    from fractura_b200 import _lib
    from fractura_b200 import batch as fb
    from fractura_b200 import dist
    from fractura_b200 import high_precision as hp

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
    with ClockSampler(local_rank) as clocks:
        time.sleep(0.3)
        torch.cuda.synchronize()
        clocks.mark(True)
        torch.cuda.nvtx.range_push("timed_region")
        step_ms = timed_loop(torch, stream, flush, steps, g.replay)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        clocks.mark(False)
    # a graph replay launches the batch kernel once; the library's counter does not see it
    launches = (L.ap_launch_counter() - c0) + steps
    barrier(world)
    total_ms = max_over_ranks(float(np.sum(step_ms)), world)
    value = dist.whole_job_rate(iters, steps, world, total_ms) / 1e9

    # end to end: orbits (host), tables and records (device), the persistent launch and
    # the download of every tile's smooth map, per step
    e2e_steps = 2 if headline else 1
    barrier(world)
    t0 = time.perf_counter()
    h2d = d2h = 0
    for _ in range(e2e_steps):
        hp.clear_reference_orbit_cache()
        # the tiles whose references are ready render while the host searches the others
        sb = fb.render_streamed(tiles, arith=wl["arith"], bla_form=wl["bla_form"], stream=stream, cfg=cfg)
        stream.synchronize()  # the maps are read once the batch stream has finished
        maps = [o["iter"].cpu() for o in sb.tiles_out]
        d2h = sum(m.numel() * 4 for m in maps)
        h2d = sum(sum(16 * (p.ref_len + 1) for p in part.params) + len(part.desc_dev) for part in sb.parts)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    barrier(world)
    e2e = iters * e2e_steps * world / e2e_s / 1e9
    forms = {}
    if rank == 0 and "One-Pass" in wl.get("glitch_mode", ""):
        # the single-reference comparator: every tile on one reference with Pauldelbrot
        # flags; pixels that outlive their tile's reference are flagged and iterated on
        # directly in FP64 from the reference's end (values not to be trusted)
        hp.clear_reference_orbit_cache()
        sw = dict(wl, glitch_mode="Off (Single-Ref)")
        b1 = fb.prepare_batch(batch_tiles(sw), arith="ref_cuda" if wl["arith"] == "fast" else wl["arith"],
                              bla_form=wl["bla_form"], stream=stream)
        b1.render(cfg)
        torch.cuda.synchronize()
        ms1 = timed_loop(torch, stream, flush, max(3, steps // 5), lambda: b1.render(cfg))
        it1 = b1.nominal_iterations()
        glitched = sum(int(o["glitch"].count_nonzero().item()) for o in b1.tiles_out)
        pixels = sum(t.W * t.H for t in b1.tiles)
        forms["single_reference"] = {
            "form": "every tile on one reference with Pauldelbrot flags, no rebasing",
            "value": it1 / (float(np.median(ms1)) * 1e-3) / 1e9, "unit": "G iter/s",
            "ms_per_batch": float(np.median(ms1)), "glitched_pixels": glitched,
            "glitched_fraction": glitched / pixels}
    if rank == 0:
        forms["fp32_floatexp"] = batch_fp32_form(torch, fb, hp, wl, b, cfg, stream, flush, steps)
    if rank != 0:
        return None
    flops = batch_flops(torch, _lib, b, cfg)
    kernel_ms = float(np.median(step_ms))  # the step is the graph's one persistent launch
    peak64 = fma_peak_tflops(64, torch)
    achieved = flops / (kernel_ms * 1e-3) / 1e12
    return {
        "metric": "G iter/s", "value": value, "unit": "G iter/s", "n_gpus": world,
        "steps": steps, "warmup": args.warmup, "ms_per_step": total_ms / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"],
        "data": "synthetic", "impl": "ours", "config": config_of(wl, world), "form": wl["form"],
        "arith": wl["arith"], "bla_form": wl["bla_form"],
        "nominal_iterations_per_batch": iters,
        "roofline": {"bound": "fp64", "kernel": "batch_kernel (one persistent launch per step)",
                     "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                     "frac": achieved / peak64 if peak64 else None,
                     "peak_source": "measured dependent-FMA FP64 probe (ap_fma_peak_launch), this run",
                     "kernel_ms_per_step": kernel_ms, "traffic": None},
        "e2e": {"value": e2e, "unit": "G iter/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                "path": "batch.render_streamed (host orbits; each time the device is idle, the tiles ready so "
                        "far get their tables and go to one launch) + download of every tile",
                "launches_per_step": len(sb.parts)},
        "forms": forms,
        "autotuner": {"chosen": vars(cfg) if hasattr(cfg, "__dict__") else repr(cfg),
                      "candidates_ms": [[round(ms, 4), repr(c)] for ms, c in fb.tuned_timings(b)]},
        "clocks": clocks.summary(),
        "gpu_launches": int(launches),
    }


# ------------------------------------------------------------ adjoint arm
def adjoint_arm(args, wl, rank, world, local_rank, steps, headline):
    """Config 5: per step, for Julia and Multibrot n=3, the forward pass with checkpoints,
    the loss gradient dL/ds on the device and the adjoint sweep (the autograd backward);
    value = forward orbit iterations per second (each iteration is also swept backwards)."""
    import torch
    from fractura_b200 import _lib
    from fractura_b200 import adjoint as adj
    from fractura_b200 import dist

    stream = torch.cuda.Stream()
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")
    L = _lib.load()
    W, H, mi = wl["W"], wl["H"], wl["max_iter"]
    rng = np.random.default_rng(wl["seed"])
    cases = []
    for case in wl["cases"]:
        th = np.array(case["theta"], np.float64)
        tgt_th = th + rng.normal(0.0, 1e-3, size=5)
        with torch.cuda.stream(stream):
            tgt, _, _ = adj.forward(tgt_th.tolist(), W, H, mi, case["fractal_type"], case["gen_n"], ckpt=False)
        stream.synchronize()
        cases.append((case, th, tgt))

    def one_step(timing=None):
        out = []
        for case, th, tgt in cases:
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)] if timing is not None else None
            if ev:
                ev[0].record(torch.cuda.current_stream())
            s, k, ck = adj.forward(th.tolist(), W, H, mi, case["fractal_type"], case["gen_n"])
            g = torch.where((s >= 0) & (tgt >= 0), 2.0 * (s - tgt), torch.zeros_like(s)) / float(W * H)
            if ev:
                ev[1].record(torch.cuda.current_stream())
            out.append((adj.adjoint(th.tolist(), g, k, ck, W, H, mi, case["fractal_type"], case["gen_n"]), k))
            if ev:
                ev[2].record(torch.cuda.current_stream())
                timing.append(ev)
        return out

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            res = one_step()
        evs = []
        one_step(evs)
    stream.synchronize()
    fwd_ms = sum(e[0].elapsed_time(e[1]) for e in evs)
    adj_ms = sum(e[1].elapsed_time(e[2]) for e in evs)
    iters = fwd_flops = adj_flops = 0.0
    for (case, _, _), (_, k) in zip(cases, res):
        it = nominal_iterations(k.cpu().numpy(), mi)
        iters += it
        if case["fractal_type"] == 4:
            fwd_flops += flops_fwd_multi(case["gen_n"]) * it
            adj_flops += flops_adj_multi(case["gen_n"]) * it
        else:
            fwd_flops += FLOPS_FWD_QUAD * it
            adj_flops += FLOPS_ADJ_QUAD * it

    barrier(world)
    c0 = L.ap_launch_counter()
    with ClockSampler(local_rank) as clocks:
        time.sleep(0.3)
        torch.cuda.synchronize()
        clocks.mark(True)
        torch.cuda.nvtx.range_push("timed_region")
        step_ms = timed_loop(torch, stream, flush, steps, one_step)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        clocks.mark(False)
    launches = L.ap_launch_counter() - c0
    barrier(world)
    total_ms = max_over_ranks(float(np.sum(step_ms)), world)
    value = dist.whole_job_rate(iters, steps, world, total_ms) / 1e9

    # end to end through the autograd Function: the target image comes from pinned host
    # memory each step, the loss and the gradient go back
    tgt_host = [tgt.cpu().pin_memory() for _, _, tgt in cases]
    e2e_steps = max(3, steps // 10)

    def e2e_step():
        for (case, th, _), th_host in zip(cases, tgt_host):
            theta = torch.tensor(th, dtype=torch.float64, device="cuda", requires_grad=True)
            tg = th_host.to("cuda", non_blocking=True)
            s = adj.smooth_escape(theta, W, H, mi, case["fractal_type"], case["gen_n"])
            mask = (s >= 0) & (tg >= 0)
            loss = torch.where(mask, (s - tg) ** 2, torch.zeros_like(s)).mean()
            loss.backward()
            _ = float(loss.item()), theta.grad.cpu().numpy()

    e2e_step()  # warm-up: the autograd path's first call is not timed
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    barrier(world)
    e2e = iters * e2e_steps * world / e2e_s / 1e9
    if rank != 0:
        return None
    peak64 = fma_peak_tflops(64, torch)
    achieved = adj_flops / (adj_ms * 1e-3) / 1e12
    return {
        "metric": "G iter/s", "value": value, "unit": "G iter/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": total_ms / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"], "data": "synthetic", "impl": "ours",
        "config": config_of(wl, world), "form": wl["form"],
        "nominal_iterations_per_step": iters,
        "kernel_ms": {"forward": fwd_ms, "adjoint": adj_ms},
        "flops_per_step": {"forward": fwd_flops, "adjoint": adj_flops,
                           "per_iteration": {"forward_quadratic": FLOPS_FWD_QUAD,
                                             "adjoint_quadratic": FLOPS_ADJ_QUAD,
                                             "forward_multibrot3": flops_fwd_multi(3),
                                             "adjoint_multibrot3": flops_adj_multi(3)}},
        "roofline": {"bound": "fp64", "kernel": "smooth_adjoint_kernel (the larger of the two)",
                     "achieved": achieved, "peak": peak64, "unit": "TFLOP/s",
                     "frac": achieved / peak64 if peak64 else None,
                     "forward_frac": (fwd_flops / (fwd_ms * 1e-3) / 1e12) / peak64 if peak64 else None,
                     "peak_source": "measured dependent-FMA FP64 probe (ap_fma_peak_launch), this run",
                     "kernel_ms_per_step": adj_ms, "traffic": None},
        "e2e": {"value": e2e, "unit": "G iter/s",
                "h2d_bytes_per_step": int(sum(t.numel() * 8 for t in tgt_host) + 2 * 5 * 8),
                "d2h_bytes_per_step": int(2 * (5 * 8 + 8)), "steps": e2e_steps,
                "path": "adjoint.smooth_escape (torch.autograd.Function) forward + loss.backward()"},
        "clocks": clocks.summary(),
        "gpu_launches": int(launches),
    }


# -------------------------------------------------------------------- main
def run_workload(args, wl, rank, world, local_rank, steps, headline):
    kind = wl.get("kind")
    if kind == "batch":
        return batch_arm(args, wl, rank, world, local_rank, steps, headline)
    if kind == "adjoint":
        return adjoint_arm(args, wl, rank, world, local_rank, steps, headline)
    return frame_arm(args, wl, rank, world, local_rank, steps, headline)


def cpu_budget(wl, headline):
    if wl.get("kind") == "batch":
        return 8.0
    return 12.0 if headline else 4.0


SUB_KEYS = ("metric", "value", "unit", "steps", "ms_per_step", "config", "form", "arith", "bla_form",
            "roofline", "e2e", "cpu_baseline", "forms", "clocks", "gpu_launches", "kernel_ms",
            "flops_per_step", "autotuner", "nominal_iterations_per_frame", "nominal_iterations_per_batch",
            "nominal_iterations_per_step", "rebase_passes", "work_per_frame")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--configs", default="auto", choices=["auto", "none"],
                    help="auto: with the default workload on one GPU, also measure every other config")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank, world, local_rank = dist_env()
    wl = WORKLOADS[args.workload]()
    if args.impl == "reference":
        cpu_reference_arm(args, wl, rank, world)
        return
    import torch
    torch.cuda.set_device(local_rank)
    if world > 1:
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=timedelta(seconds=120))
    try:
        line = run_workload(args, wl, rank, world, local_rank, args.steps, True)
        if rank == 0:
            line["cpu_baseline"] = cpu_baseline_record(wl, cpu_budget(wl, True))
        if args.configs == "auto" and args.workload == DEFAULT_WORKLOAD and world == 1:
            line["configs"] = {}
            for name in SUB_RECORDS:
                sw = WORKLOADS[name]()
                sub = run_workload(args, sw, rank, world, local_rank, min(args.steps, 20), False)
                sub["cpu_baseline"] = cpu_baseline_record(sw, cpu_budget(sw, False))
                line["configs"][name] = {k: sub[k] for k in SUB_KEYS if k in sub}
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch.distributed as tdist
            tdist.destroy_process_group()


if __name__ == "__main__":
    main()
