"""Generate the golden fixtures under tests/golden/ by running the reference.

Run where the reference's source tree is available, with APEIRON_REFERENCE_ROOT set to
it (the directory holding config.py and math_core/):

    APEIRON_REFERENCE_ROOT=<reference tree> python tests/golden/make_golden.py [section ...]

Every fixture records the inputs it was made from, so the tests rebuild the
same inputs without the reference.  Sections:

  fp64     per-sample FP64 escape values for all five formulas
           (math_core/cpu_kernels.py:228 cpu_compute_fp64_sample)
  render1  full-frame renders of the 640x360 Mandelbrot overview through
           math_core/engine.py:471 render_frame_cpu (schemes 0..11, SSAA)
  dd       per-sample double-double escape values
           (math_core/cpu_kernels.py:271 cpu_compute_dd_sample)
  render2  Burning Ship DD frames at 1e-20 with 2x adaptive SSAA
  orbits   Decimal reference orbits (math_core/high_precision.py:706)
  pert     per-sample FP64-delta perturbation values with and without
           chained BLA (math_core/cpu_kernels.py:374)
  bla      chained-BLA tables (math_core/high_precision.py:1101)
  fexp     FloatExp perturbation samples at 1e-1000
           (math_core/cpu_kernels.py:606)
  render3  deep-zoom perturbation frames with Pauldelbrot rebasing
  probe    adaptive max-iter probe maps and depths (math_core/engine.py:1063)
"""
import hashlib
import json
import math
import os
import sys
import time
from decimal import Decimal

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ref_shim  # noqa: E402

R = ref_shim.install()
INV_LN2 = R.config.INV_LN2_F32
LN_BAIL = R.config.LN_BAILOUT_LOG

SEED = 20261203


def save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"  wrote {name}: {os.path.getsize(path) / 1024:.1f} KiB")


# ---------------------------------------------------------------------------
# Per-sample FP64 escape values
# ---------------------------------------------------------------------------
FP64_CASES = [
    # name, fractal_type, cx, cy, width, max_iter, jx, jy, n, kr, ki
    ("mandel_seahorse", 0, -0.7436439, 0.1318259, 1e-6, 2000, 0.0, 0.0, 3, 0.25, 1.0),
    ("mandel_overview", 0, -0.65, 0.0, 4.0, 500, 0.0, 0.0, 3, 0.25, 1.0),
    ("ship", 1, -1.75, 0.03, 0.18, 1000, 0.0, 0.0, 3, 0.25, 1.0),
    ("julia", 2, 0.0, 0.0, 3.0, 2000, -0.8, 0.156, 3, 0.25, 1.0),
    ("ship_julia", 3, 0.0, 0.0, 4.0, 1000, -1.755, 0.03, 3, 0.25, 1.0),
    ("multibrot3", 4, 0.0, 0.0, 3.0, 1000, 0.0, 0.0, 3, 0.1, 0.2),
    ("multibrot4", 4, 0.0, 0.0, 3.0, 1000, 0.0, 0.0, 4, 0.1, 0.2),
    ("multibrot5", 4, 0.0, 0.0, 3.0, 600, 0.0, 0.0, 5, 0.1, 0.2),
    ("multibrot2k", 4, -0.5, 0.0, 3.0, 800, 0.0, 0.0, 2, 0.25, 1.0),
]
FP64_W, FP64_H = 128, 72


def fp64_grid(cx, cy, w):
    """Plain IEEE grid: x = x_min + i*dx, y = y_max - j*dy (no contraction)."""
    h = w * FP64_H / FP64_W
    dx = w / (FP64_W - 1)
    dy = h / (FP64_H - 1)
    x_min = cx - w * 0.5
    y_max = cy + h * 0.5
    i = np.arange(FP64_W, dtype=np.float64)
    j = np.arange(FP64_H, dtype=np.float64)
    xs = x_min + i * dx
    ys = y_max - j * dy
    return xs, ys


def gen_fp64():
    out = {}
    meta = []
    f = R.ck.cpu_compute_fp64_sample
    for (name, ft, cx, cy, w, mi, jx, jy, n, kr, ki) in FP64_CASES:
        xs, ys = fp64_grid(cx, cy, w)
        s = np.empty((FP64_H, FP64_W), np.float32)
        for jj in range(FP64_H):
            for ii in range(FP64_W):
                s[jj, ii] = f(float(xs[ii]), float(ys[jj]), mi, ft, jx, jy, n, kr, ki, INV_LN2, LN_BAIL)
        out[name + "__s"] = s
        out[name + "__x"] = xs
        out[name + "__y"] = ys
        meta.append(dict(name=name, fractal_type=ft, max_iter=mi, julia_cx=jx, julia_cy=jy,
                         gen_n=n, gen_kr=kr, gen_ki=ki))
    save("fp64_samples.npz", meta=json.dumps(meta), **out)


# ---------------------------------------------------------------------------
# Full-frame FP64 renders through render_frame_cpu
# ---------------------------------------------------------------------------
RENDER1_CASES = [
    # name, W, H, max_iter, cx, cy, width, scheme, factor, offset, density, contrast, type, jx, jy, n, kr, ki
    ("cfg1_hist", 640, 360, 1000, "-0.65", "0.0", "4.0", 11, 1, 0.0, 1.0, 1.0, 0, 0.0, 0.0, 3, 0.25, 1.0),
    ("cfg1_s0", 640, 360, 1000, "-0.65", "0.0", "4.0", 0, 1, 0.0, 1.0, 1.0, 0, 0.0, 0.0, 3, 0.25, 1.0),
    ("ssaa2_s0", 160, 90, 500, "-0.7436", "0.1318", "0.02", 0, 2, 0.0, 1.0, 1.0, 0, 0.0, 0.0, 3, 0.25, 1.0),
    ("ssaa2_hist", 160, 90, 500, "-0.7436", "0.1318", "0.02", 11, 2, 0.1, 1.3, 0.8, 0, 0.0, 0.0, 3, 0.25, 1.0),
    ("ssaa3_julia", 96, 54, 400, "0.0", "0.0", "3.0", 6, 3, 0.2, 1.0, 1.0, 2, -0.8, 0.156, 3, 0.25, 1.0),
] + [
    (f"scheme{sid}", 96, 54, 600, "-0.7436", "0.1318", "0.05", sid, 1, 0.15 * (sid % 3), 1.0 + 0.1 * sid,
     1.0 if sid % 2 == 0 else 1.4, 0, 0.0, 0.0, 3, 0.25, 1.0)
    for sid in range(1, 11)
] + [
    ("ship_s2", 96, 54, 300, "-1.75", "0.03", "0.18", 2, 1, 0.0, 1.0, 1.0, 1, 0.0, 0.0, 3, 0.25, 1.0),
    ("multibrot_s5", 96, 54, 300, "0.0", "0.0", "3.0", 5, 2, 0.3, 0.7, 1.2, 4, 0.0, 0.0, 3, 0.1, 0.2),
    ("shipjulia_hist", 96, 54, 300, "0.0", "0.0", "4.0", 11, 1, 0.0, 1.0, 1.0, 3, -1.755, 0.03, 3, 0.25, 1.0),
]


def gen_render1():
    out = {}
    meta = []
    for c in RENDER1_CASES:
        (name, W, H, mi, cx, cy, w, sid, fac, off, den, con, ft, jx, jy, n, kr, ki) = c
        it = np.zeros((H, W), np.float32)
        t0 = time.time()
        rgb = R.engine.render_frame_cpu(
            W, H, mi, Decimal(cx), Decimal(cy), Decimal(w), "synthetic",
            ssaa_factor=fac, edge_threshold=0.35, color_scheme_id=sid,
            precision_mode="1e-12 (FP64)", fractal_type=ft, julia_cx=jx, julia_cy=jy,
            bbsa_tol=1e-4, bbsa_order=4, glitch_mode="Off (Single-Ref)",
            gen_n=n, gen_kr=kr, gen_ki=ki, cpu_threads=8, palette_offset=off,
            color_density=den, color_contrast=con, h_iter_buf=it)
        print(f"  {name}: {time.time() - t0:.2f}s")
        out[name + "__rgb"] = rgb
        out[name + "__iter"] = it
        meta.append(dict(name=name, W=W, H=H, max_iter=mi, cx=cx, cy=cy, width=w, scheme=sid,
                         factor=fac, offset=off, density=den, contrast=con, fractal_type=ft,
                         julia_cx=jx, julia_cy=jy, gen_n=n, gen_kr=kr, gen_ki=ki))
    save("render_fp64.npz", meta=json.dumps(meta), **out)


def config2_centre(seed=SEED):
    """Config-2 centre: (-1.75 + 1e-17*u1, 0.03 + 1e-17*u2), u ~ U(-1, 1) from the seed."""
    rng = np.random.default_rng(seed)
    u1, u2 = rng.uniform(-1.0, 1.0, size=2)
    cx = Decimal("-1.75") + Decimal(repr(float(u1))) * Decimal("1e-17")
    cy = Decimal("0.03") + Decimal(repr(float(u2))) * Decimal("1e-17")
    return str(cx), str(cy)


def render2_cases():
    cx2, cy2 = config2_centre()
    return [
        # Burning Ship DD at 1e-20, 2x adaptive SSAA (config 2 at quarter size).
        ("cfg2_quarter", 320, 180, 20000, cx2, cy2, "1e-20", 0, 2, 0.0, 1.0, 1.0, 1, 0.0, 0.0, 3, 0.25, 1.0),
        ("cfg2_hist", 160, 90, 20000, cx2, cy2, "1e-20", 11, 2, 0.0, 1.0, 1.0, 1, 0.0, 0.0, 3, 0.25, 1.0),
        ("dd_mandel", 64, 36, 3000, "-0.10109636384562", "0.95628651080914", "4e-18", 0, 1,
         0.0, 1.0, 1.0, 0, 0.0, 0.0, 3, 0.25, 1.0),
        ("dd_mandel_ssaa", 48, 27, 3000, "-0.10109636384562", "0.95628651080914", "3e-17", 6, 2,
         0.1, 1.0, 1.0, 0, 0.0, 0.0, 3, 0.25, 1.0),
        ("dd_julia", 64, 36, 2000, "0.123456789012345678", "0.0987654321098765", "1e-16", 0, 1,
         0.0, 1.0, 1.0, 2, -0.8, 0.156, 3, 0.25, 1.0),
        ("dd_shipjulia", 64, 36, 2000, "0.1", "0.2", "1e-15", 0, 1, 0.0, 1.0, 1.0, 3, -1.755, 0.03,
         3, 0.25, 1.0),
        ("dd_multibrot3", 64, 36, 2000, "-0.5641", "0.6612", "1e-14", 0, 1, 0.0, 1.0, 1.0, 4, 0.0, 0.0,
         3, 0.1, 0.2),
        ("dd_multibrot5", 48, 27, 1000, "0.7", "0.2", "1e-13", 11, 1, 0.0, 1.0, 1.0, 4, 0.0, 0.0,
         5, 0.1, 0.2),
    ]


def gen_render2():
    out = {}
    meta = []
    for c in render2_cases():
        (name, W, H, mi, cx, cy, w, sid, fac, off, den, con, ft, jx, jy, n, kr, ki) = c
        it = np.zeros((H, W), np.float32)
        t0 = time.time()
        rgb = R.engine.render_frame_cpu(
            W, H, mi, Decimal(cx), Decimal(cy), Decimal(w), "synthetic",
            ssaa_factor=fac, edge_threshold=0.35, color_scheme_id=sid,
            precision_mode="1e-24 (DD)", fractal_type=ft, julia_cx=jx, julia_cy=jy,
            bbsa_tol=1e-4, bbsa_order=4, glitch_mode="Off (Single-Ref)",
            gen_n=n, gen_kr=kr, gen_ki=ki, cpu_threads=8, palette_offset=off,
            color_density=den, color_contrast=con, h_iter_buf=it)
        print(f"  {name}: {time.time() - t0:.2f}s  escaped {np.mean(it >= 0):.3f}")
        out[name + "__rgb"] = rgb
        out[name + "__iter"] = it
        meta.append(dict(name=name, W=W, H=H, max_iter=mi, cx=cx, cy=cy, width=w, scheme=sid,
                         factor=fac, offset=off, density=den, contrast=con, fractal_type=ft,
                         julia_cx=jx, julia_cy=jy, gen_n=n, gen_kr=kr, gen_ki=ki))
    save("render_dd.npz", meta=json.dumps(meta), **out)


# ---------------------------------------------------------------------------
# Deep-zoom workloads (config 3): preset centre extended with seeded digits
# ---------------------------------------------------------------------------
def config3_centre(seed=SEED, digits=600):
    """The 1e-160 preset centre (presets.json:154-157) extended to `digits` decimals."""
    with open(os.path.join(ref_shim.REF_ROOT, "presets.json")) as f:
        data = json.load(f)
    marks = data.get("bookmarks", data) if isinstance(data, dict) else data
    e = next(b for b in marks if "1e-160" in b.get("name", "") and b.get("fractal_type") == 0)
    rng = np.random.default_rng(seed)
    out = []
    for key in ("center_x", "center_y"):
        v = e[key]
        frac = v.split(".")[1]
        extra = "".join(str(d) for d in rng.integers(0, 10, size=max(0, digits - len(frac))))
        out.append(v + extra)
    return out[0], out[1]


def write_workloads():
    cx3, cy3 = config3_centre()
    cx2, cy2 = config2_centre()
    path = os.path.join(HERE, "workloads.json")
    wl = json.load(open(path)) if os.path.exists(path) else {}
    wl.update({"seed": SEED, "config2_centre": [cx2, cy2], "config3_centre": [cx3, cy3]})
    with open(os.path.join(HERE, "workloads.json"), "w") as f:
        json.dump(wl, f, indent=1)
    print("  wrote workloads.json")
    return wl


def deep_point(ft, cx, cy, w, jx=0.0, jy=0.0, n=3, kr=0.25, ki=1.0, levels=6, grid=96, mi=3000):
    """Deterministic boundary search: zoom x40 per level toward the escaped grid point
    with the largest escape value (reference FP64 evaluator)."""
    f = R.ck.cpu_compute_fp64_sample
    for _ in range(levels):
        best = (-1.0, cx, cy)
        for jj in range(grid):
            y = cy + w * (0.5 - jj / (grid - 1))
            for ii in range(grid):
                x = cx + w * (ii / (grid - 1) - 0.5)
                v = f(x, y, mi, ft, jx, jy, n, kr, ki, INV_LN2, LN_BAIL)
                if v > best[0]:
                    best = (float(v), x, y)
        _, cx, cy = best
        w /= 40.0
    return repr(cx), repr(cy)


PERT_SPECS = [
    # name, fractal_type, start cx, cy, width, W, H, max_iter, stride, jx, jy, n, kr, ki
    ("ship", 1, -1.75, -0.03, 0.2, 640, 360, 6000, 10, 0.0, 0.0, 3, 0.25, 1.0),
    ("julia", 2, 0.0, 0.0, 3.0, 640, 360, 6000, 10, -0.8, 0.156, 3, 0.25, 1.0),
    ("ship_julia", 3, 0.0, 0.0, 4.0, 640, 360, 6000, 10, -1.755, 0.03, 3, 0.25, 1.0),
    ("multibrot3", 4, 0.0, 0.0, 3.0, 640, 360, 6000, 10, 0.0, 0.0, 3, 0.1, 0.2),
    ("multibrot4", 4, 0.0, 0.0, 3.0, 320, 180, 6000, 8, 0.0, 0.0, 4, 0.1, 0.2),
]


def pert_cases():
    cases = [("cfg3", 0, None, None, "1e-160", 1920, 1080, 200000, 40, 0.0, 0.0, 3, 0.25, 1.0)]
    for (name, ft, cx, cy, w, W, H, mi, stride, jx, jy, n, kr, ki) in PERT_SPECS:
        px, py = deep_point(ft, cx, cy, w, jx, jy, n, kr, ki)
        cases.append((name, ft, px, py, "2e-14", W, H, mi, stride, jx, jy, n, kr, ki))
    return cases


def gen_pert():
    wl = write_workloads()
    hp, ck, cfg = R.hp, R.ck, R.config
    out = {}
    meta = []
    for (name, ft, cx, cy, w, W, H, mi, stride, jx, jy, n, kr, ki) in pert_cases():
        if cx is None:
            cx, cy = wl["config3_centre"]
        cfg.ensure_decimal_precision(Decimal(w))
        pw = Decimal(w)
        ph = pw * (Decimal(H) / Decimal(W))
        hp.clear_reference_orbit_cache()
        t0 = time.time()
        bcx, bcy, bu, bv, re, im, rl = hp.find_optimal_reference_orbit(
            Decimal(cx), Decimal(cy), pw, ph, mi, W, H, fractal_type=ft, julia_cx=jx, julia_cy=jy,
            gen_n=n, gen_kr=kr, gen_ki=ki, is_floatexp=False)
        t_orbit = time.time() - t0
        dx = float(pw / Decimal(max(1, W - 1)))
        dy = float(ph / Decimal(max(1, H - 1)))
        ref_px = float(W - 1) * float(bu)
        ref_py = float(H - 1) * float(bv)
        tab = hp.build_bla_table(re, im, rl, fractal_type=ft, tol=1e-6, gen_n=n, gen_kr=kr, gen_ki=ki)
        zero16 = (0.0,) * 16
        si = np.arange(0, W, stride, dtype=np.float64)
        sj = np.arange(0, H, stride, dtype=np.float64)
        res = {}
        for variant, table, strict in (("plain", np.zeros((1, 1, 1)), 0), ("bla", tab, 1)):
            s = np.empty((len(sj), len(si)), np.float32)
            g = np.empty((len(sj), len(si)), np.uint8)
            for a, jj in enumerate(sj):
                for b, ii in enumerate(si):
                    sv, gl = ck.cpu_compute_perturbation_sample(
                        re, im, rl, mi, ref_px, ref_py, float(ii), float(jj), dx, dy,
                        float(bcx), float(bcy), ft, float(jx), float(jy), 0, 1.0, *zero16,
                        n, kr, ki, strict, INV_LN2, LN_BAIL, bla_table=table)
                    s[a, b] = sv
                    g[a, b] = gl
            res[variant] = (s, g)
        print(f"  {name}: ref_len {rl} at u,v=({bu},{bv}) orbit {t_orbit:.1f}s total {time.time()-t0:.1f}s "
              f"glitched(bla) {res['bla'][1].mean():.3f}")
        out[name + "__re"] = re[:rl + 1]
        out[name + "__im"] = im[:rl + 1]
        for variant in res:
            out[f"{name}__{variant}_s"] = res[variant][0]
            out[f"{name}__{variant}_g"] = res[variant][1]
        out[name + "__bla_sha256"] = np.frombuffer(
            hashlib.sha256(np.ascontiguousarray(tab).tobytes()).digest(), np.uint8)
        meta.append(dict(name=name, fractal_type=ft, cx=cx, cy=cy, width=w, W=W, H=H, max_iter=mi,
                         stride=stride, julia_cx=jx, julia_cy=jy, gen_n=n, gen_kr=kr, gen_ki=ki,
                         ref_cx=str(bcx), ref_cy=str(bcy), u=bu, v=bv, ref_len=int(rl),
                         bla_shape=list(tab.shape), dx=dx, dy=dy, ref_px=ref_px, ref_py=ref_py))
    save("pert_samples.npz", meta=json.dumps(meta), **out)


def gen_bbsa():
    """Series-approximation starts: compute_bbsa_coeffs (math_core/high_precision.py:537) on
    the perturbation goldens' orbits, orders 4 and 8, and per-sample values that start from
    them (cpu_compute_perturbation_sample, no BLA)."""
    hp, ck, cfg = R.hp, R.ck, R.config
    G = np.load(os.path.join(HERE, "pert_samples.npz"))
    pmeta = json.loads(str(G["meta"]))
    out = {}
    meta = []
    for m in pmeta:
        name, ft = m["name"], m["fractal_type"]
        if ft not in (0, 2, 4):
            continue
        re, im, rl = G[name + "__re"], G[name + "__im"], m["ref_len"]
        max_r = float(Decimal(m["width"])) * 0.75
        for order in (4, 8):
            for tol in (1e-4, 1e-6):
                tag = f"{name}__o{order}_t{int(-math.log10(tol))}"
                res = hp.compute_bbsa_coeffs(re, im, rl, max_r, ft, bbsa_tol=tol, bbsa_order=order,
                                             gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"],
                                             E_scale=0)
                coeffs = np.array(res, np.float64)
                out[tag + "__coeffs"] = coeffs
                meta.append(dict(name=name, tag=tag, order=order, tol=tol, max_r=max_r,
                                 skip=int(res[0])))
                if tol != 1e-4:
                    continue
                st = m["stride"] * 2
                si = np.arange(0, m["W"], st, dtype=np.float64)
                sj = np.arange(0, m["H"], st, dtype=np.float64)
                sv = np.empty((len(sj), len(si)), np.float32)
                for a, jj in enumerate(sj):
                    for b, ii in enumerate(si):
                        sv[a, b], _ = ck.cpu_compute_perturbation_sample(
                            re, im, rl, m["max_iter"], m["ref_px"], m["ref_py"], float(ii), float(jj),
                            m["dx"], m["dy"], float(Decimal(m["ref_cx"])), float(Decimal(m["ref_cy"])), ft,
                            float(m["julia_cx"]), float(m["julia_cy"]), int(res[0]), 1.0 / max_r,
                            *res[1:17], m["gen_n"], m["gen_kr"], m["gen_ki"], 0, INV_LN2, LN_BAIL,
                            bla_table=np.zeros((1, 1, 1)))
                out[tag + "__s"] = sv
                out[tag + "__stride"] = np.array([st])
                print(f"  {tag}: skip {int(res[0])} escaped {np.mean(sv >= 0):.3f}")
    save("bbsa_samples.npz", meta=json.dumps(meta), **out)


def gen_render_bbsa():
    """Frames with series-approximation starts (bbsa_order 4 and 8, tol 1e-4) through
    render_frame_cpu, Pauldelbrot rebasing on."""
    G = np.load(os.path.join(HERE, "pert_samples.npz"))
    pm = {m["name"]: m for m in json.loads(str(G["meta"]))}
    out = {}
    meta = []
    for (name, src, order, W, H, gm) in (("bbsa4_cfg3", "cfg3", 4, 160, 90, "Pauldelbrot"),
                                         ("bbsa8_cfg3", "cfg3", 8, 160, 90, "Off (Single-Ref)"),
                                         ("bbsa4_julia", "julia", 4, 160, 90, "Pauldelbrot"),
                                         ("bbsa8_multibrot3", "multibrot3", 8, 160, 90, "Off (Single-Ref)")):
        m = pm[src]
        mi = min(m["max_iter"], 20000)
        R.hp.clear_reference_orbit_cache()
        it = np.zeros((H, W), np.float32)
        t0 = time.time()
        rgb = R.engine.render_frame_cpu(
            W, H, mi, Decimal(m["cx"]), Decimal(m["cy"]), Decimal(m["width"]), "synthetic",
            ssaa_factor=1, edge_threshold=0.35, color_scheme_id=0,
            precision_mode="1e-300 (Perturbation)", fractal_type=m["fractal_type"],
            julia_cx=m["julia_cx"], julia_cy=m["julia_cy"], bbsa_tol=1e-4, bbsa_order=order,
            glitch_mode=gm, gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"], cpu_threads=8,
            palette_offset=0.0, color_density=1.0, color_contrast=1.0, h_iter_buf=it)
        print(f"  {name}: {time.time() - t0:.2f}s escaped {np.mean(it >= 0):.3f}")
        out[name + "__rgb"] = rgb
        out[name + "__iter"] = it
        meta.append(dict(name=name, W=W, H=H, max_iter=mi, cx=m["cx"], cy=m["cy"], width=m["width"],
                         scheme=0, factor=1, bbsa_order=order, bbsa_tol=1e-4, glitch_mode=gm,
                         fractal_type=m["fractal_type"], julia_cx=m["julia_cx"], julia_cy=m["julia_cy"],
                         gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"]))
    save("render_bbsa.npz", meta=json.dumps(meta), **out)


FEXP_SPECS = [
    # name, fractal_type, width, W, H, max_iter, stride, jx, jy, n, kr, ki  (centre: the pert case's)
    ("fexp_mandel", 0, "1e-320", 480, 270, 20000, 10, 0.0, 0.0, 3, 0.25, 1.0),
    ("fexp_ship", 1, "1e-320", 480, 270, 6000, 10, 0.0, 0.0, 3, 0.25, 1.0),
    ("fexp_julia", 2, "1e-400", 480, 270, 6000, 10, -0.8, 0.156, 3, 0.25, 1.0),
    ("fexp_multibrot3", 4, "1e-320", 480, 270, 6000, 10, 0.0, 0.0, 3, 0.1, 0.2),
]


def fexp_cases():
    wl = json.load(open(os.path.join(HERE, "workloads.json")))
    pc = {c[0]: c for c in pert_cases()}
    src = {0: "cfg3", 1: "ship", 2: "julia", 4: "multibrot3"}
    cases = []
    for (name, ft, w, W, H, mi, stride, jx, jy, n, kr, ki) in FEXP_SPECS:
        c = pc[src[ft]]
        cx, cy = (c[2], c[3]) if c[2] is not None else tuple(wl["config3_centre"])
        cases.append((name, ft, cx, cy, w, W, H, mi, stride, jx, jy, n, kr, ki))
    cx3, cy3 = wl["config3_centre"]
    # config 3 at 1e-1000 (the reference's FloatExp tier), every 60th pixel
    cases.append(("fexp_cfg3", 0, cx3, cy3, "1e-1000", 1920, 1080, 20000, 60, 0.0, 0.0, 3, 0.25, 1.0))
    return cases


def gen_fexp():
    """Per-sample FloatExp perturbation values (cpu_compute_perturbation_sample_floatexp)."""
    hp, ck, cfg = R.hp, R.ck, R.config
    out = {}
    meta = []
    for (name, ft, cx, cy, w, W, H, mi, stride, jx, jy, n, kr, ki) in fexp_cases():
        cfg.ensure_decimal_precision(Decimal(w))
        pw = Decimal(w)
        ph = pw * (Decimal(H) / Decimal(W))
        E = cfg.compute_floatexp_scale(pw)
        hp.clear_reference_orbit_cache()
        t0 = time.time()
        bcx, bcy, bu, bv, re, im, rl = hp.find_optimal_reference_orbit(
            Decimal(cx), Decimal(cy), pw, ph, mi, W, H, fractal_type=ft, julia_cx=jx, julia_cy=jy,
            gen_n=n, gen_kr=kr, gen_ki=ki, is_floatexp=True)
        t_orbit = time.time() - t0
        two_e = Decimal(2) ** E
        dx = float(pw * two_e / Decimal(max(1, W - 1)))
        dy = float(ph * two_e / Decimal(max(1, H - 1)))
        ref_px = float(W - 1) * float(bu)
        ref_py = float(H - 1) * float(bv)
        tab = hp.build_bla_table(re, im, rl, fractal_type=ft, tol=1e-6, gen_n=n, gen_kr=kr, gen_ki=ki)
        zero16 = (0.0,) * 16
        si = np.arange(0, W, stride, dtype=np.float64)
        sj = np.arange(0, H, stride, dtype=np.float64)
        res = {}
        for variant, table, strict in (("plain", np.zeros((1, 1, 1)), 0), ("bla", tab, 1)):
            s = np.empty((len(sj), len(si)), np.float32)
            g = np.empty((len(sj), len(si)), np.uint8)
            for a, jj in enumerate(sj):
                for b, ii in enumerate(si):
                    sv, gl = ck.cpu_compute_perturbation_sample_floatexp(
                        re, im, rl, mi, ref_px, ref_py, float(ii), float(jj), dx, dy, E,
                        float(bcx), float(bcy), ft, float(jx), float(jy), 0, 1.0, *zero16,
                        n, kr, ki, strict, INV_LN2, LN_BAIL, bla_table=table)
                    s[a, b] = sv
                    g[a, b] = gl
            res[variant] = (s, g)
        print(f"  {name}: E {E} ref_len {rl} orbit {t_orbit:.1f}s total {time.time() - t0:.1f}s "
              f"escaped {np.mean(res['plain'][0] >= 0):.3f} glitched(bla) {res['bla'][1].mean():.3f}")
        out[name + "__re"] = re[:rl + 1]
        out[name + "__im"] = im[:rl + 1]
        for variant in res:
            out[f"{name}__{variant}_s"] = res[variant][0]
            out[f"{name}__{variant}_g"] = res[variant][1]
        meta.append(dict(name=name, fractal_type=ft, cx=cx, cy=cy, width=w, W=W, H=H, max_iter=mi,
                         stride=stride, julia_cx=jx, julia_cy=jy, gen_n=n, gen_kr=kr, gen_ki=ki,
                         ref_cx=str(bcx), ref_cy=str(bcy), u=bu, v=bv, ref_len=int(rl), e_scale=int(E),
                         bla_shape=list(tab.shape), dx=dx, dy=dy, ref_px=ref_px, ref_py=ref_py))
    save("fexp_samples.npz", meta=json.dumps(meta), **out)


CONFIG4_FORMULAS = [
    # fractal_type, julia (jx, jy), gen_n, kr, ki
    (0, (0.0, 0.0), 3, 0.25, 1.0),
    (1, (0.0, 0.0), 3, 0.25, 1.0),
    (2, (-0.8, 0.156), 3, 0.25, 1.0),
    (3, (-1.755, 0.03), 3, 0.25, 1.0),
    (4, (0.0, 0.0), 3, 0.1, 0.2),
    (4, (0.0, 0.0), 4, 0.1, 0.2),
    (4, (0.0, 0.0), 5, 0.1, 0.2),
]


def _escape_count(fx, x, y, n_iter, bits):
    ft, (jx, jy), n, kr, ki = fx
    from fractura_b200 import high_precision as hp
    return int(hp.compute_highprec_escape_scalar(x, y, n_iter, ft, jx, jy, bits, n, kr, ki))


def gen_config4():
    """Config 4: 64 seeded square tiles -- edge U{64..512}, formula uniform over the seven of
    CONFIG4_FORMULAS, max_iter = floor(10^U(3,5)), width 10^U(-60,-12) -- centred on
    boundary points.  Per tile: the point of a 48 x 48 grid over [-2, 2]^2 with the most
    escape steps (at most N = min(max_iter, 2000)) is the inner end, a point 3 away
    along a seeded ray the outer end, and the bracket is bisected on "at least as many
    escape steps as the inner end" (the set's boundary when the inner end stays bounded
    for N steps, else a level curve of the escape time) until it is below a quarter of
    the width, with the engine's native escape test at the tile's orbit precision.
    Written into workloads.json."""
    from fractura_b200.config import compute_required_prec_bits
    rng = np.random.default_rng(SEED + 4)
    path = os.path.join(HERE, "workloads.json")
    wl = json.load(open(path))
    tiles = []
    t0 = time.time()
    grid = [Decimal(repr(-2.0 + 4.0 * q / 47.0)) for q in range(48)]
    inner_cache = {}
    for q in range(64):
        fi = int(rng.integers(0, len(CONFIG4_FORMULAS)))
        fx = CONFIG4_FORMULAS[fi]
        edge = int(rng.integers(64, 513))
        W = H = edge
        max_iter = int(10 ** rng.uniform(3, 5))
        width = Decimal(repr(float(10 ** rng.uniform(-60, -12)))).normalize()
        theta = float(rng.uniform(0.0, 2.0 * math.pi))
        bits = compute_required_prec_bits(width)
        n_test = min(max_iter, 2000)
        key = (fi, n_test)
        if key not in inner_cache:
            best = (-1, None)
            for y in grid:
                for x in grid:
                    e = _escape_count(fx, x, y, n_test, 128)
                    if e > best[0]:
                        best = (e, (x, y))
            inner_cache[key] = best
        level, inner = inner_cache[key]
        with __import__("decimal").localcontext() as ctx:
            ctx.prec = int(-width.adjusted()) + 40
            lo = inner
            hi = (lo[0] + Decimal(repr(3.0 * math.cos(theta))), lo[1] + Decimal(repr(3.0 * math.sin(theta))))
            while max(abs(hi[0] - lo[0]), abs(hi[1] - lo[1])) > width / 4:
                mid = ((lo[0] + hi[0]) / 2, (lo[1] + hi[1]) / 2)
                if _escape_count(fx, mid[0], mid[1], n_test, bits) >= level:
                    lo = mid
                else:
                    hi = mid
            cx, cy = (lo[0] + hi[0]) / 2, (lo[1] + hi[1]) / 2
        ft, (jx, jy), n, kr, ki = fx
        tiles.append(dict(cx=str(cx), cy=str(cy), width=str(width), W=W, H=H, max_iter=max_iter,
                          fractal_type=ft, julia_cx=jx, julia_cy=jy, gen_n=n, gen_kr=kr, gen_ki=ki))
        print(f"  tile {q}: type {ft} n {n} {W}x{H} max_iter {max_iter} width {width} "
              f"(inner level {level}) {time.time() - t0:.0f}s", flush=True)
    wl["config4_tiles"] = tiles
    wl["config4_seed"] = SEED + 4
    with open(path, "w") as f:
        json.dump(wl, f, indent=1)
    px = sum(t["W"] * t["H"] for t in tiles)
    print(f"  config 4: {len(tiles)} tiles, {px} pixels, {time.time() - t0:.0f}s")


def render3_cases():
    wl = json.load(open(os.path.join(HERE, "workloads.json")))
    cx3, cy3 = wl["config3_centre"]
    pc = {c[0]: c for c in pert_cases()}
    cases = [
        # name, W, H, max_iter, cx, cy, width, scheme, factor, bbsa_order, glitch_mode, type, jx, jy, n, kr, ki
        ("cfg3_bla_pauldelbrot", 192, 108, 20000, cx3, cy3, "1e-160", 0, 1, 32, "Pauldelbrot", 0, 0.0, 0.0, 3, 0.25, 1.0),
        ("cfg3_plain", 192, 108, 20000, cx3, cy3, "1e-160", 5, 1, 0, "Off (Single-Ref)", 0, 0.0, 0.0, 3, 0.25, 1.0),
        ("cfg3_hist", 128, 72, 20000, cx3, cy3, "1e-160", 11, 1, 32, "Pauldelbrot", 0, 0.0, 0.0, 3, 0.25, 1.0),
        ("cfg3_ssaa2", 64, 36, 20000, cx3, cy3, "1e-160", 0, 2, 32, "Pauldelbrot", 0, 0.0, 0.0, 3, 0.25, 1.0),
        ("cfg3_hist_ssaa2", 64, 36, 20000, cx3, cy3, "1e-160", 11, 2, 32, "Pauldelbrot", 0, 0.0, 0.0, 3, 0.25, 1.0),
    ]
    for name in ("ship", "julia", "ship_julia", "multibrot3"):
        c = pc[name]
        cases.append((f"{name}_frame", 160, 90, c[7], c[2], c[3], c[4], 0, 1, 32, "Pauldelbrot",
                      c[1], c[9], c[10], c[11], c[12], c[13]))
    return cases


def gen_render3():
    out = {}
    meta = []
    for c in render3_cases():
        (name, W, H, mi, cx, cy, w, sid, fac, order, gm, ft, jx, jy, n, kr, ki) = c
        R.hp.clear_reference_orbit_cache()
        it = np.zeros((H, W), np.float32)
        t0 = time.time()
        rgb = R.engine.render_frame_cpu(
            W, H, mi, Decimal(cx), Decimal(cy), Decimal(w), "synthetic",
            ssaa_factor=fac, edge_threshold=0.35, color_scheme_id=sid,
            precision_mode="1e-300 (Perturbation)", fractal_type=ft, julia_cx=jx, julia_cy=jy,
            bbsa_tol=1e-6 if order == 32 else 0.0, bbsa_order=order, glitch_mode=gm,
            gen_n=n, gen_kr=kr, gen_ki=ki, cpu_threads=8, palette_offset=0.0,
            color_density=1.0, color_contrast=1.0, h_iter_buf=it)
        print(f"  {name}: {time.time() - t0:.2f}s escaped {np.mean(it >= 0):.3f}")
        out[name + "__rgb"] = rgb
        out[name + "__iter"] = it
        meta.append(dict(name=name, W=W, H=H, max_iter=mi, cx=cx, cy=cy, width=w, scheme=sid,
                         factor=fac, bbsa_order=order, glitch_mode=gm, fractal_type=ft,
                         julia_cx=jx, julia_cy=jy, gen_n=n, gen_kr=kr, gen_ki=ki,
                         offset=0.0, density=1.0, contrast=1.0))
    save("render_pert.npz", meta=json.dumps(meta), **out)


def strict_cases():
    pc = {c[0]: c for c in pert_cases()}
    cases = []
    # name, source case, W, H, max_iter, scheme
    for (name, src, W, H, mi, sid) in (("strict_ship", "ship", 48, 27, 1500, 0),
                                       ("strict_julia_hist", "julia", 48, 27, 1500, 11),
                                       ("strict_ship_julia", "ship_julia", 48, 27, 1500, 5),
                                       ("strict_multibrot3", "multibrot3", 48, 27, 1500, 0)):
        c = pc[src]
        cases.append((name, W, H, mi, c[2], c[3], c[4], sid, 1, 32, "Strict Metric",
                      c[1], c[9], c[10], c[11], c[12], c[13]))
    return cases


def gen_strict():
    """Strict Metric frames through render_frame_cpu: rebasing stops at 128 glitched
    pixels or after 4 passes, then every pixel still flagged is evaluated on its own
    high-precision orbit (math_core/engine.py:191-267, :1033-1046)."""
    out = {}
    meta = []
    for c in strict_cases():
        (name, W, H, mi, cx, cy, w, sid, fac, order, gm, ft, jx, jy, n, kr, ki) = c
        R.hp.clear_reference_orbit_cache()
        it = np.zeros((H, W), np.float32)
        t0 = time.time()
        rgb = R.engine.render_frame_cpu(
            W, H, mi, Decimal(cx), Decimal(cy), Decimal(w), "synthetic",
            ssaa_factor=fac, edge_threshold=0.35, color_scheme_id=sid,
            precision_mode="1e-300 (Perturbation)", fractal_type=ft, julia_cx=jx, julia_cy=jy,
            bbsa_tol=1e-6, bbsa_order=order, glitch_mode=gm,
            gen_n=n, gen_kr=kr, gen_ki=ki, cpu_threads=8, palette_offset=0.0,
            color_density=1.0, color_contrast=1.0, h_iter_buf=it)
        print(f"  {name}: {time.time() - t0:.2f}s escaped {np.mean(it >= 0):.3f}")
        out[name + "__rgb"] = rgb
        out[name + "__iter"] = it
        meta.append(dict(name=name, W=W, H=H, max_iter=mi, cx=cx, cy=cy, width=w, scheme=sid,
                         factor=fac, bbsa_order=order, glitch_mode=gm, fractal_type=ft,
                         julia_cx=jx, julia_cy=jy, gen_n=n, gen_kr=kr, gen_ki=ki,
                         offset=0.0, density=1.0, contrast=1.0))
    save("render_strict.npz", meta=json.dumps(meta), **out)


# ---------------------------------------------------------------------------
# Adaptive max-iter probe (math_core/engine.py:1063-1281, CPU branch)
# ---------------------------------------------------------------------------
def probe_cases():
    wl = json.load(open(os.path.join(HERE, "workloads.json")))
    cx3, cy3 = wl["config3_centre"]
    cx2, cy2 = wl["config2_centre"]
    pc = {c[0]: c for c in pert_cases()}
    P, DD = "1e-300 (Perturbation)", "1e-24 (DD)"
    cases = [
        # name, cx, cy, width, base_iter, W, H, type, jx, jy, n, kr, ki, precision, bbsa_tol, bbsa_order
        ("fp64_overview", "-0.65", "0.0", "3.0", 500, 128, 72, 0, 0.0, 0.0, 3, 0.25, 1.0, P, 1e-4, 4),
        ("fp64_ship", "-1.75", "-0.03", "0.2", 400, 128, 72, 1, 0.0, 0.0, 3, 0.25, 1.0, P, 1e-4, 4),
        ("fp64_multibrot4", "0.0", "0.0", "3.0", 300, 96, 54, 4, 0.0, 0.0, 4, 0.1, 0.2, P, 1e-4, 4),
        ("dd_ship", cx2, cy2, "1e-20", 3000, 64, 36, 1, 0.0, 0.0, 3, 0.25, 1.0, DD, 1e-4, 4),
        ("dd_mandel", "-0.10109636384562", "0.95628651080914", "4e-18", 1500, 64, 36, 0, 0.0, 0.0, 3, 0.25,
         1.0, DD, 1e-4, 4),
        ("pert_cfg3", cx3, cy3, "1e-160", 10000, 64, 36, 0, 0.0, 0.0, 3, 0.25, 1.0, P, 1e-4, 4),
    ]
    # No FloatExp view: the reference's CPU FloatExp probe kernel
    # (math_core/cpu_kernels.py:1087) fails to compile in Numba ("Calling a closure
    # with *args is unsupported"), so that branch raises; its device kernel is
    # pinned in the CUDA simulator instead (make_golden_cudasim.py).
    for (name, order, tol) in (("julia", 4, 1e-4), ("ship_julia", 4, 1e-4), ("multibrot3", 4, 1e-4),
                               ("ship", 8, 1e-6)):
        c = pc[name]
        cases.append((f"pert_{name}", c[2], c[3], c[4], 3000, 64, 36, c[1], c[9], c[10], c[11], c[12], c[13],
                      P, tol, order))
    return cases


def gen_probe():
    """The reference's probe (probe_adaptive_max_iter with compute_device='CPU') on
    views of every tier; its probe map is recorded where it hands it to
    get_adaptive_max_iter_from_probe, with the depth it returns."""
    E = R.engine
    seen = []
    orig = E.get_adaptive_max_iter_from_probe

    def record(iters, base):
        seen.append(np.array(iters, np.float32, copy=True))
        return orig(iters, base)

    E.get_adaptive_max_iter_from_probe = record
    out = {}
    meta = []
    try:
        for c in probe_cases():
            (name, cx, cy, w, base, W, H, ft, jx, jy, n, kr, ki, prec, tol, order) = c
            R.hp.clear_reference_orbit_cache()
            seen.clear()
            t0 = time.time()
            depth = E.probe_adaptive_max_iter(
                Decimal(cx), Decimal(cy), Decimal(w), base, target_w=W, target_h=H, fractal_type=ft,
                julia_cx=jx, julia_cy=jy, gen_n=n, gen_kr=kr, gen_ki=ki, precision_mode=prec,
                bbsa_tol=tol, bbsa_order=order, compute_device="CPU", cpu_threads=8)
            assert len(seen) == 1
            print(f"  {name}: {time.time() - t0:.2f}s depth {depth} escaped {np.mean(seen[0] >= 0):.3f}")
            out[name + "__iter"] = seen[0]
            meta.append(dict(name=name, cx=cx, cy=cy, width=w, base_iter=base, W=W, H=H, fractal_type=ft,
                             julia_cx=jx, julia_cy=jy, gen_n=n, gen_kr=kr, gen_ki=ki, precision_mode=prec,
                             bbsa_tol=tol, bbsa_order=order, depth=int(depth)))
    finally:
        E.get_adaptive_max_iter_from_probe = orig
    save("probe.npz", meta=json.dumps(meta), **out)


# ---------------------------------------------------------------------------
# Ground truth for precision checks: direct iteration in 700-bit arithmetic
# (mpmath), independent of the reference and of perturbation theory.
# ---------------------------------------------------------------------------
LN_BAIL_CONFIG = 1.7129177284488854  # config.py:26 of the reference


def _truth_row(args):
    import mpmath
    (cx, cy, width, W, H, cols, row, mi, bits) = args
    mpmath.mp.prec = bits
    pw = mpmath.mpf(width)
    ph = pw * H / W
    x_min = mpmath.mpf(cx) - pw / 2
    y_max = mpmath.mpf(cy) + ph / 2
    y = y_max - ph * row / (H - 1)
    out = []
    big = mpmath.mpf(65536)
    # The smooth term uses the reference's hard-coded LN_BAILOUT_LOG (config.py:26,
    # 1.09e-5 below ln(0.5 ln 65536)) that its render passes use, so that only the
    # escape dynamics differ.
    ln_bailout = mpmath.mpf(LN_BAIL_CONFIG)
    for col in cols:
        x = x_min + pw * col / (W - 1)
        zx = zy = mpmath.mpf(0)
        val = -1.0
        for k in range(mi):
            zx2, zy2 = zx * zx, zy * zy
            m2 = zx2 + zy2
            if m2 > big:
                lm = mpmath.log(m2)
                val = float(k + 1 - (mpmath.log(lm / 2) - ln_bailout) / mpmath.log(2))
                break
            zy = 2 * zx * zy + y
            zx = zx2 - zy2 + x
        out.append(val)
    return out


def gen_truth():
    from multiprocessing import get_context
    wl = json.load(open(os.path.join(HERE, "workloads.json")))
    cx, cy = wl["config3_centre"]
    W, H, mi = 1920, 1080, 20000
    cols = list(range(0, W, 30))
    rows = list(range(0, H, 17))
    t0 = time.time()
    with get_context("spawn").Pool(os.cpu_count()) as pool:
        res = pool.map(_truth_row, [(cx, cy, "1e-160", W, H, cols, r, mi, 700) for r in rows])
    truth = np.array(res, dtype=np.float64)
    print(f"  truth {truth.shape} in {time.time() - t0:.0f}s, escaped {np.mean(truth >= 0):.3f}")
    save("truth_cfg3.npz", s=truth, cols=np.array(cols), rows=np.array(rows),
         meta=json.dumps(dict(width="1e-160", W=W, H=H, max_iter=mi, bits=700,
                              note="direct z^2+c iteration in 700-bit mpmath at the exact pixel c; smooth term with the reference's LN_BAILOUT_LOG constant")))


SECTIONS = {"truth": gen_truth, "fp64": gen_fp64, "render1": gen_render1, "render2": gen_render2, "pert": gen_pert,
            "fexp": gen_fexp, "bbsa": gen_bbsa, "render_bbsa": gen_render_bbsa, "config4": gen_config4,
            "render3": gen_render3, "strict": gen_strict,
            "probe": gen_probe}

if __name__ == "__main__":
    wanted = sys.argv[1:] or list(SECTIONS)
    for s in wanted:
        print(f"[{s}]")
        SECTIONS[s]()
