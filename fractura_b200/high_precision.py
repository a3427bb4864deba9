"""Host-side high-precision inputs of the perturbation tiers.

Restates math_core/high_precision.py's reference-orbit machinery with the
reference's Decimal arithmetic (its path when gmpy2 is absent,
math_core/high_precision.py:657-703 and :802-873), so the orbit arrays are
bit-identical to the reference's:

  compute_single_highprec_orbit   math_core/high_precision.py:706-875
  compute_highprec_escape_scalar  math_core/high_precision.py:581-703
  find_optimal_reference_orbit    math_core/high_precision.py:919-1097
  cache_reference_orbit / clear_reference_orbit_cache (16-entry LRU)

Every computation runs in a local Decimal context; the caller's context is
never modified.
"""
import math
import os
import threading
from concurrent.futures import ThreadPoolExecutor
from decimal import Decimal, localcontext

import numpy as np

from .config import INV_LN2_F32, LN_BAILOUT_LOG, compute_required_prec_bits, decimal_context

_ORBIT_CACHE = []
_ORBIT_LOCK = threading.Lock()
_CACHE_SIZE = 16


def _orbit_context(prec_bits):
    ctx = decimal_context()
    ctx.prec = int(prec_bits / 3.32) + 30
    return ctx


def _start(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy):
    if fractal_type in (2, 3):
        return (Decimal(cand_cx), Decimal(cand_cy), Decimal(str(julia_cx)), Decimal(str(julia_cy)))
    return Decimal(0), Decimal(0), Decimal(cand_cx), Decimal(cand_cy)


def _step(fractal_type, zx, zy, zx2, zy2, c_x, c_y, two, n, kr, ki):
    """One Decimal iteration, in the reference's operation order."""
    if fractal_type in (0, 2):
        return zx2 - zy2 + c_x, two * zx * zy + c_y
    if fractal_type in (1, 3):
        return zx2 - zy2 + c_x, two * abs(zx) * abs(zy) - c_y
    zn_r, zn_i = zx, zy
    for _ in range(n - 1):
        zn_r, zn_i = zn_r * zx - zn_i * zy, zn_r * zy + zn_i * zx
    kz_r = kr * zx - ki * zy
    kz_i = kr * zy + ki * zx
    return zn_r + kz_r + c_x, zn_i + kz_i + c_y


def compute_single_highprec_orbit(cand_cx_dec, cand_cy_dec, max_iter, fractal_type=0,
                                  julia_cx=0.0, julia_cy=0.0, prec_bits=256,
                                  gen_n=3, gen_kr=0.25, gen_ki=1.0):
    """Reference orbit Z_0..Z_ref_len as float64 arrays of length max_iter + 1.

    ref_len is the step at which |Z|^2 > 65536 in Decimal arithmetic (max_iter
    if it never does).  For Mandelbrot and its Julia set an exactly repeating
    orbit is detected at power-of-two checkpoints and its cycle is copied to
    the end of the arrays.
    """
    ref_re = np.zeros(max_iter + 1, dtype=np.float64)
    ref_im = np.zeros(max_iter + 1, dtype=np.float64)
    with localcontext(_orbit_context(prec_bits)):
        bailout = Decimal(65536)
        two = Decimal(2)
        zx, zy, c_x, c_y = _start(fractal_type, cand_cx_dec, cand_cy_dec, julia_cx, julia_cy)
        kr, ki = Decimal(str(gen_kr)), Decimal(str(gen_ki))
        ref_len = max_iter
        periodic = fractal_type in (0, 2)
        check_step, saved_k = 8, 0
        saved_x, saved_y = zx, zy
        for k in range(max_iter):
            ref_re[k], ref_im[k] = float(zx), float(zy)
            zx2, zy2 = zx * zx, zy * zy
            if (zx2 + zy2) > bailout:
                ref_len = k
                break
            if periodic:
                if k == check_step:
                    check_step <<= 1
                    saved_k = k
                    saved_x, saved_y = zx, zy
                elif k > saved_k and zx == saved_x and zy == saved_y:
                    period = k - saved_k
                    if period > 0:
                        for j in range(k, max_iter + 1):
                            ref_re[j] = ref_re[j - period]
                            ref_im[j] = ref_im[j - period]
                        return ref_re, ref_im, max_iter
            zx, zy = _step(fractal_type, zx, zy, zx2, zy2, c_x, c_y, two, gen_n, kr, ki)
        ref_re[ref_len], ref_im[ref_len] = float(zx), float(zy)
    return ref_re, ref_im, ref_len


def compute_highprec_escape_scalar(cand_cx, cand_cy, max_iter, fractal_type=0,
                                   julia_cx=0.0, julia_cy=0.0, prec_bits=256,
                                   gen_n=3, gen_kr=0.25, gen_ki=1.0):
    """Smooth escape value of one point in Decimal arithmetic (max_iter if it stays bounded)."""
    with localcontext(_orbit_context(prec_bits)):
        bailout = Decimal(65536)
        two = Decimal(2)
        zx, zy, c_x, c_y = _start(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy)
        kr, ki = Decimal(str(gen_kr)), Decimal(str(gen_ki))
        inv_n = (1.0 / math.log(float(gen_n))) if (fractal_type == 4 and gen_n > 1) else float(INV_LN2_F32)
        for k in range(max_iter):
            zx2, zy2 = zx * zx, zy * zy
            mag2_dec = zx2 + zy2
            if mag2_dec > bailout:
                log_mag = math.log(float(mag2_dec))
                if log_mag > 1.0:
                    return float(k + 1.0) - (math.log(0.5 * log_mag) - LN_BAILOUT_LOG) * inv_n
                return float(k)
            zx, zy = _step(fractal_type, zx, zy, zx2, zy2, c_x, c_y, two, gen_n, kr, ki)
        return float(max_iter)


def clear_reference_orbit_cache():
    """Drop every cached reference orbit."""
    with _ORBIT_LOCK:
        _ORBIT_CACHE.clear()


def cache_reference_orbit(cx_dec, cy_dec, pw_dec, max_iter, ref_re, ref_im, ref_len,
                          fractal_type=0, julia_cx=0.0, julia_cy=0.0,
                          gen_n=3, gen_kr=0.25, gen_ki=1.0, is_floatexp=False):
    """Insert an orbit at the front of the 16-entry LRU (math_core/high_precision.py:893-916)."""
    with _ORBIT_LOCK:
        _ORBIT_CACHE.insert(0, dict(is_floatexp=is_floatexp, fractal_type=fractal_type,
                                    julia_cx=julia_cx, julia_cy=julia_cy, gen_n=gen_n,
                                    gen_kr=gen_kr, gen_ki=gen_ki, pw_dec=pw_dec, cx_dec=cx_dec,
                                    cy_dec=cy_dec, ref_len=ref_len, max_iter=max_iter,
                                    ref_re=ref_re, ref_im=ref_im))
        if len(_ORBIT_CACHE) > _CACHE_SIZE:
            _ORBIT_CACHE.pop()


PROBE_UV = [
    (0.35, 0.35), (0.65, 0.35), (0.35, 0.65), (0.65, 0.65),
    (0.5, 0.25), (0.5, 0.75), (0.25, 0.5), (0.75, 0.5),
    (0.2, 0.2), (0.8, 0.2), (0.2, 0.8), (0.8, 0.8),
    (0.5, 0.35), (0.5, 0.65), (0.35, 0.5), (0.65, 0.5),
]


def find_optimal_reference_orbit(cx_dec, cy_dec, pw_dec, ph_dec, max_iter, screen_w, screen_h,
                                 fractal_type=0, julia_cx=0.0, julia_cy=0.0,
                                 gen_n=3, gen_kr=0.25, gen_ki=1.0, is_floatexp=False):
    """Reference orbit for a view: cached, at the centre, or at the best of 16 probes.

    Returns (cx_dec, cy_dec, u, v, ref_re, ref_im, ref_len) where (u, v) is the
    reference's position in the view as fractions of its width and height
    (math_core/high_precision.py:919-1097).
    """
    ctx = decimal_context(pw_dec)
    with localcontext(ctx):
        x_min_dec = cx_dec - (pw_dec / Decimal(2))
        y_max_dec = cy_dec + (ph_dec / Decimal(2))
        best_entry, best_score = None, -1
        with _ORBIT_LOCK:
            for e in _ORBIT_CACHE:
                if e.get("is_floatexp", False) != is_floatexp:
                    continue
                if (e["fractal_type"] == fractal_type and e["julia_cx"] == julia_cx and
                        e["julia_cy"] == julia_cy and e["gen_n"] == gen_n and
                        e["gen_kr"] == gen_kr and e["gen_ki"] == gen_ki):
                    ratio = pw_dec / e["pw_dec"]
                    if Decimal("0.25") <= ratio <= Decimal("4.0"):
                        cu = float((e["cx_dec"] - x_min_dec) / pw_dec)
                        cv = float((y_max_dec - e["cy_dec"]) / ph_dec)
                        if 0.10 <= cu <= 0.90 and 0.10 <= cv <= 0.90 and e["ref_len"] > best_score:
                            best_score = e["ref_len"]
                            best_entry = e
                            if e["ref_len"] >= max_iter:
                                break
            can_reuse = False
            if best_entry is not None:
                entry_max = best_entry.get("max_iter", best_entry["ref_len"])
                natural = best_entry["ref_len"] < entry_max
                ratio = pw_dec / best_entry["pw_dec"]
                panning = Decimal("0.75") <= ratio <= Decimal("1.33")
                if best_score >= max_iter:
                    can_reuse = True
                elif panning and best_score >= 100 and (best_entry["ref_len"] >= max_iter or natural):
                    can_reuse = True
                elif natural and best_score >= int(max_iter * 0.35):
                    can_reuse = True
                elif (best_entry["cx_dec"] == cx_dec and best_entry["cy_dec"] == cy_dec and
                      best_entry["pw_dec"] == pw_dec and (best_entry["ref_len"] >= max_iter or natural)):
                    can_reuse = True
            if can_reuse and best_entry is not None:
                u = float((best_entry["cx_dec"] - x_min_dec) / pw_dec)
                v = float((y_max_dec - best_entry["cy_dec"]) / ph_dec)
                return (best_entry["cx_dec"], best_entry["cy_dec"], u, v, best_entry["ref_re"],
                        best_entry["ref_im"], min(best_entry["ref_len"], max_iter))

        bits = compute_required_prec_bits(pw_dec)
        ref_re, ref_im, ref_len = compute_single_highprec_orbit(
            cx_dec, cy_dec, max_iter, fractal_type, julia_cx, julia_cy, bits,
            gen_n=gen_n, gen_kr=gen_kr, gen_ki=gen_ki)
        best_cx, best_cy, best_u, best_v = cx_dec, cy_dec, 0.5, 0.5

        if ref_len < int(max_iter * 0.6) and pw_dec >= Decimal("1e-10000"):
            def probe(uv):
                u, v = uv
                with localcontext(ctx):
                    cand_x = x_min_dec + Decimal(str(u)) * pw_dec
                    cand_y = y_max_dec - Decimal(str(v)) * ph_dec
                esc = compute_highprec_escape_scalar(cand_x, cand_y, max_iter, fractal_type,
                                                     julia_cx, julia_cy, bits, gen_n, gen_kr, gen_ki)
                return esc, cand_x, cand_y, u, v

            workers = min(len(PROBE_UV), os.cpu_count() or 4)
            with ThreadPoolExecutor(max_workers=workers) as ex:
                results = list(ex.map(probe, PROBE_UV))
            best_esc = max(int(ref_len * 1.2), ref_len + 32)
            cand = (cx_dec, cy_dec, 0.5, 0.5)
            for esc, cand_x, cand_y, u, v in results:
                if esc > best_esc:
                    best_esc = esc
                    cand = (cand_x, cand_y, u, v)
            if cand[0] != cx_dec or cand[1] != cy_dec:
                c_re, c_im, c_len = compute_single_highprec_orbit(
                    cand[0], cand[1], max_iter, fractal_type, julia_cx, julia_cy, bits,
                    gen_n=gen_n, gen_kr=gen_kr, gen_ki=gen_ki)
                if c_len > ref_len:
                    ref_re, ref_im, ref_len = c_re, c_im, c_len
                    best_cx, best_cy, best_u, best_v = cand

        if can_reuse and best_entry is not None and best_entry["ref_len"] > ref_len:
            u = float((best_entry["cx_dec"] - x_min_dec) / pw_dec)
            v = float((y_max_dec - best_entry["cy_dec"]) / ph_dec)
            return (best_entry["cx_dec"], best_entry["cy_dec"], u, v, best_entry["ref_re"],
                    best_entry["ref_im"], min(best_entry["ref_len"], max_iter))

        cache_reference_orbit(best_cx, best_cy, pw_dec, max_iter, ref_re, ref_im, ref_len,
                              fractal_type, julia_cx, julia_cy, gen_n, gen_kr, gen_ki, is_floatexp)
        return best_cx, best_cy, best_u, best_v, ref_re, ref_im, ref_len
