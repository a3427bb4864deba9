"""Golden fixtures of the reference's CUDA-only Strict Metric fallback, made by running
its Numba CUDA kernels in Numba's CUDA simulator (NUMBA_ENABLE_CUDASIM=1) on the CPU.

    python tests/golden/make_golden_cudasim.py

Writes ``strict_cuda.npz``:

  ml_*     compute_ml_sample (math_core/cuda_kernels.py:2372-2446) at seeded points of
           all four fixed-point formulas, with the limbs decimal_to_limbs (:2242-2274)
           made for them;
  frame_*  eval_glitched_pixels_fallback_cuda (math_core/engine.py:270-410) on listed
           pixels of small views: the double-double tier (1e-20, with and without the
           histogram colouring) and the fixed-point tier (1e-34), each recording the
           iteration map, RGB and glitch map it leaves.

The simulator runs the kernels' Python source with IEEE arithmetic, so the fixtures
hold the kernels' source semantics; the compiled kernels are fastmath, which permits
reassociation the simulator does not do.  The simulator's cuda.fma is an unfused
a * b + c, which would zero the double-double error-free products; it is replaced here
by a correctly rounded fused multiply-add (exact rational arithmetic), the device's.
"""
import json
import math
import os
import sys
import time
from decimal import Decimal, getcontext
from fractions import Fraction

os.environ["NUMBA_ENABLE_CUDASIM"] = "1"

import numpy as np  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ref_shim  # noqa: E402

R = ref_shim.install()
from math_core import cuda_kernels as K  # noqa: E402
from numba import cuda  # noqa: E402
from numba.cuda.simulator import kernelapi  # noqa: E402

E = R.engine
E.HAS_CUDA = True  # device-array pool of the reference, backed by the simulator


def _fused_fma(self, a, b, c):
    if not (math.isfinite(a) and math.isfinite(b) and math.isfinite(c)):
        return a * b + c
    return float(Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c)))


kernelapi.FakeCUDAModule.fma = _fused_fma
SEED = 20261203
JULIA = {2: (-0.8, 0.156), 3: (-1.755, 0.03)}


@cuda.jit
def _ml_kernel(out, sx, lx, sy, ly, max_iter, ft, jxs, jxl, jys, jyl):
    if cuda.grid(1) == 0:
        out[0] = K.compute_ml_sample(sx, lx, sy, ly, max_iter, ft, jxs, jxl, jys, jyl)


def _fp64_escape(ft, x, y, jx, jy, mi):
    zx, zy, cx, cy = (x, y, jx, jy) if ft in (2, 3) else (0.0, 0.0, x, y)
    for k in range(mi):
        if ft in (1, 3):
            zx, zy = abs(zx), abs(zy)
        if zx * zx + zy * zy >= 65536.0:
            return k
        zx, zy = zx * zx - zy * zy + cx, (2.0 * zx * zy - cy) if ft in (1, 3) else (2.0 * zx * zy + cy)
    return mi


def gen_ml_points(per_type=24, max_iter=160):
    rng = np.random.default_rng(SEED)
    getcontext().prec = 500
    rows = []
    out = np.zeros(1, np.float32)
    zero = np.zeros(K.ML_LIMBS, np.uint32)
    for ft in (0, 1, 2, 3):
        jx, jy = JULIA.get(ft, (0.0, 0.0))
        jxs, jxl = K.decimal_to_limbs(Decimal(str(jx))) if ft in (2, 3) else (0, zero)
        jys, jyl = K.decimal_to_limbs(Decimal(str(jy))) if ft in (2, 3) else (0, zero)
        n = 0
        while n < per_type:
            # 40 random digits: every fraction limb of the fixed-point c is in play
            x = Decimal(int(rng.integers(-2_200_000, 1_000_000))) / Decimal(1_000_000) + \
                Decimal(int(rng.integers(0, 10 ** 17))) * Decimal("1e-40")
            y = Decimal(int(rng.integers(-1_500_000, 1_500_000))) / Decimal(1_000_000) - \
                Decimal(int(rng.integers(0, 10 ** 17))) * Decimal("1e-40")
            k = _fp64_escape(ft, float(x), float(y), jx, jy, max_iter)
            if k < 2 or (k >= max_iter and rng.random() > 0.1):
                continue
            sx, lx = K.decimal_to_limbs(x)
            sy, ly = K.decimal_to_limbs(y)
            _ml_kernel[1, 1](out, sx, lx, sy, ly, max_iter, ft, jxs, jxl, jys, jyl)
            rows.append(dict(ft=ft, x=str(x), y=str(y), jx=jx, jy=jy, max_iter=max_iter, s=float(out[0]),
                             sx=int(sx), sy=int(sy), lx=[int(v) for v in lx], ly=[int(v) for v in ly]))
            n += 1
        print(f"  ml type {ft}: {n} points")
    return rows


def _frame(name, ft, cx, cy, w, W, H, mi, jx, jy, scheme, n_pix, rng, gen=(3, 0.25, 1.0)):
    lut = np.ascontiguousarray(ref_shim.synthetic_lut(2048, False), np.float32)
    d_rgb = cuda.to_device(np.zeros((H, W, 3), np.uint8))
    gl = np.zeros((H, W), np.uint8)
    flat = rng.choice(W * H, size=n_pix, replace=False)
    gl.flat[flat] = 1
    d_gl = cuda.to_device(gl)
    d_it = cuda.to_device(np.full((H, W), -7.0, np.float32))
    d_lut = cuda.to_device(lut)
    cdf = None
    d_cdf = None
    if scheme == 11:
        cdf = np.sort(rng.random(65536)).astype(np.float32)
        d_cdf = cuda.to_device(cdf)
    idx = np.argwhere(gl > 0)
    pw = Decimal(w)
    ph = pw * (Decimal(H) / Decimal(W))
    E.ensure_decimal_precision(pw)
    t0 = time.time()
    E.eval_glitched_pixels_fallback_cuda(
        d_rgb, d_gl, d_lut, idx, W, H, mi, Decimal(cx), Decimal(cy), pw, ph, scheme, ft, jx, jy,
        gen_n=gen[0], gen_kr=gen[1], gen_ki=gen[2], d_cdf_lut=d_cdf,
        num_bins=65536 if scheme == 11 else 2048, d_iter_map=d_it)
    it = d_it.copy_to_host()
    print(f"  {name}: {len(idx)} pixels {time.time() - t0:.1f}s, values {np.unique(it[gl > 0]).size} distinct")
    meta = dict(name=name, fractal_type=ft, cx=cx, cy=cy, width=w, W=W, H=H, max_iter=mi, julia_cx=jx,
                julia_cy=jy, scheme=scheme, gen_n=gen[0], gen_kr=gen[1], gen_ki=gen[2])
    arrays = {f"frame_{name}__iter": it, f"frame_{name}__rgb": d_rgb.copy_to_host(),
              f"frame_{name}__glitch_in": gl, f"frame_{name}__glitch_out": d_gl.copy_to_host()}
    if cdf is not None:
        arrays[f"frame_{name}__cdf"] = cdf
    return meta, arrays


def gen_frames():
    G = np.load(os.path.join(HERE, "pert_samples.npz"))
    pm = {m["name"]: m for m in json.loads(str(G["meta"]))}
    rng = np.random.default_rng(SEED + 1)
    metas, arrays = [], {}
    specs = [
        # name, source point, width, W, H, max_iter, scheme, listed pixels
        ("dd_ship", "ship", "1e-20", 24, 16, 6000, 0, 40),
        ("dd_julia_hist", "julia", "1e-20", 24, 16, 6000, 11, 40),
        ("dd_multibrot3", "multibrot3", "1e-20", 24, 16, 3000, 0, 24),
        ("ml_julia", "julia", "1e-34", 16, 12, 120, 0, 12),
        ("ml_ship_julia", "ship_julia", "1e-34", 16, 12, 120, 5, 12),
    ]
    for (name, src, w, W, H, mi, scheme, n_pix) in specs:
        m = pm[src]
        meta, arr = _frame(name, m["fractal_type"], m["cx"], m["cy"], w, W, H, mi, m["julia_cx"],
                           m["julia_cy"], scheme, n_pix, rng, gen=(m["gen_n"], m["gen_kr"], m["gen_ki"]))
        metas.append(meta)
        arrays.update(arr)
    return metas, arrays


if __name__ == "__main__":
    t0 = time.time()
    points = gen_ml_points()
    metas, arrays = gen_frames()
    path = os.path.join(HERE, "strict_cuda.npz")
    np.savez_compressed(path, ml=json.dumps(points), frames=json.dumps(metas), **arrays)
    print(f"  wrote strict_cuda.npz: {os.path.getsize(path) / 1024:.1f} KiB in {time.time() - t0:.0f}s")
