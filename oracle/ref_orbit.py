"""Reference orbits for the oracle, in Python's decimal module.

TEST INFRASTRUCTURE ONLY: the oracle's own reference-orbit search, so that oracle
frames and bench.py's CPU baseline share no code with the engine (whose orbits come
from its native fixed-point code).  It restates the reference's Decimal branch, which
is the reference's path wherever gmpy2 is absent (as here):

* ``orbit``       -- compute_single_highprec_orbit, Decimal branch
                     (math_core/high_precision.py:802-873): z_0 = 0 (Julia: the pixel),
                     float(z_k) stored while |z_k|^2 <= 65536, period copy for types
                     0 and 2, context precision int(bits / 3.32) + 30 digits;
* ``escape``      -- compute_highprec_escape_scalar, Decimal branch (:657-703);
* ``find_reference`` -- find_optimal_reference_orbit (:919-1097) on an empty cache:
                     the centre's orbit, and when it survives less than 0.6 max_iter the
                     16-candidate escape probe; a candidate replaces the centre only if
                     its escape beats max(1.2 ref_len, ref_len + 32) and its full orbit
                     outlives the centre's.
* ``prec_bits`` / ``view_digits`` -- config.py:36-48 and :63-74.
"""
import math
from decimal import Decimal, localcontext

import numpy as np

LN_BAILOUT_LOG = 1.7129177284488854     # config.py:26
INV_LN2_F32 = float(np.float32(1.0 / math.log(2.0)))

CANDIDATES_UV = [
    (0.35, 0.35), (0.65, 0.35), (0.35, 0.65), (0.65, 0.65),
    (0.5, 0.25), (0.5, 0.75), (0.25, 0.5), (0.75, 0.5),
    (0.2, 0.2), (0.8, 0.2), (0.2, 0.8), (0.8, 0.8),
    (0.5, 0.35), (0.5, 0.65), (0.35, 0.5), (0.65, 0.5),
]


def prec_bits(width):
    """Binary precision of a view's orbits: int(-adjusted * log2(10)) + 128, at least 64."""
    p = Decimal(str(width))
    if p <= 0:
        return 256
    return max(64, int(-p.adjusted() * 3.321928094887362) + 128)


def view_digits(width):
    """Decimal digits of the view arithmetic: max(500, -adjusted + 150)."""
    p = Decimal(str(width))
    return max(500, -p.adjusted() + 150) if p > 0 else 500


def _step(ft, zx, zy, zx2, zy2, cx, cy, n, kr, ki):
    two = Decimal(2)
    if ft in (0, 2):
        return zx2 - zy2 + cx, two * zx * zy + cy
    if ft in (1, 3):
        return zx2 - zy2 + cx, two * abs(zx) * abs(zy) - cy
    pr, pi = zx, zy
    for _ in range(n - 1):
        pr, pi = pr * zx - pi * zy, pr * zy + pi * zx
    return pr + (kr * zx - ki * zy) + cx, pi + (kr * zy + ki * zx) + cy


def _start(ft, cx, cy, julia_cx, julia_cy):
    if ft in (2, 3):
        return cx, cy, Decimal(str(julia_cx)), Decimal(str(julia_cy))
    return Decimal(0), Decimal(0), cx, cy


def orbit(cx, cy, max_iter, ft=0, julia_cx=0.0, julia_cy=0.0, bits=256, n=3, kr=0.25, ki=1.0):
    """(re, im, ref_len): float64 orbit of max_iter + 1 entries and its escape step."""
    re = np.zeros(max_iter + 1, np.float64)
    im = np.zeros(max_iter + 1, np.float64)
    bailout = Decimal(65536)
    with localcontext() as ctx:
        ctx.prec = int(bits / 3.32) + 30
        zx, zy, c_x, c_y = _start(ft, cx, cy, julia_cx, julia_cy)
        krd, kid = Decimal(str(kr)), Decimal(str(ki))
        ref_len = max_iter
        check_step, saved_k = 8, 0
        sx, sy = zx, zy
        for k in range(max_iter):
            re[k], im[k] = float(zx), float(zy)
            zx2, zy2 = zx * zx, zy * zy
            if zx2 + zy2 > bailout:
                ref_len = k
                break
            if ft in (0, 2):
                if k == check_step:
                    check_step <<= 1
                    saved_k = k
                    sx, sy = zx, zy
                elif k > saved_k and zx == sx and zy == sy:
                    period = k - saved_k
                    for j in range(k, max_iter + 1):
                        re[j] = re[j - period]
                        im[j] = im[j - period]
                    return re, im, max_iter
            zx, zy = _step(ft, zx, zy, zx2, zy2, c_x, c_y, n, krd, kid)
        re[ref_len], im[ref_len] = float(zx), float(zy)
    return re, im, ref_len


def escape(cx, cy, max_iter, ft=0, julia_cx=0.0, julia_cy=0.0, bits=256, n=3, kr=0.25, ki=1.0):
    """Smooth escape value of one point (float(max_iter) if it never escapes)."""
    bailout = Decimal(65536)
    inv_n = (1.0 / math.log(float(n))) if (ft == 4 and n > 1) else INV_LN2_F32
    with localcontext() as ctx:
        ctx.prec = int(bits / 3.32) + 30
        zx, zy, c_x, c_y = _start(ft, cx, cy, julia_cx, julia_cy)
        krd, kid = Decimal(str(kr)), Decimal(str(ki))
        for k in range(max_iter):
            zx2, zy2 = zx * zx, zy * zy
            mag2_dec = zx2 + zy2
            if mag2_dec > bailout:
                log_mag = math.log(float(mag2_dec))
                if log_mag > 1.0:
                    return float(k + 1.0) - (math.log(0.5 * log_mag) - LN_BAILOUT_LOG) * inv_n
                return float(k)
            zx, zy = _step(ft, zx, zy, zx2, zy2, c_x, c_y, n, krd, kid)
    return float(max_iter)


def find_reference(cx, cy, width, height, max_iter, ft=0, julia_cx=0.0, julia_cy=0.0, n=3, kr=0.25,
                   ki=1.0):
    """(ref_cx, ref_cy, u, v, re, im, ref_len) of a view, as the reference picks it on an
    empty orbit cache."""
    cx, cy, width, height = (x if isinstance(x, Decimal) else Decimal(str(x)) for x in (cx, cy, width, height))
    bits = prec_bits(width)
    kw = dict(ft=ft, julia_cx=julia_cx, julia_cy=julia_cy, bits=bits, n=n, kr=kr, ki=ki)
    with localcontext() as ctx:
        ctx.prec = view_digits(width)
        x_min = cx - (width / Decimal(2))
        y_max = cy + (height / Decimal(2))
        re, im, ref_len = orbit(cx, cy, max_iter, **kw)
        best = (cx, cy, 0.5, 0.5)
        if ref_len < int(max_iter * 0.6) and width >= Decimal("1e-10000"):
            probes = []
            for u, v in CANDIDATES_UV:
                cand_x = x_min + Decimal(str(u)) * width
                cand_y = y_max - Decimal(str(v)) * height
                probes.append((escape(cand_x, cand_y, max_iter, **kw), cand_x, cand_y, u, v))
            best_esc = max(int(ref_len * 1.2), ref_len + 32)
            pick = None
            for esc, cand_x, cand_y, u, v in probes:
                if esc > best_esc:
                    best_esc = esc
                    pick = (cand_x, cand_y, u, v)
            if pick is not None and (pick[0] != cx or pick[1] != cy):
                c_re, c_im, c_len = orbit(pick[0], pick[1], max_iter, **kw)
                if c_len > ref_len:
                    re, im, ref_len = c_re, c_im, c_len
                    best = pick
    return best[0], best[1], best[2], best[3], re, im, ref_len


def pixel_c(cx, cy, width, height, W, H, col, row):
    """Exact Decimal c of pixel (row, col) as the rebase loop forms a new reference
    (math_core/engine.py:1997-2006)."""
    with localcontext() as ctx:
        ctx.prec = view_digits(width)
        x_min = cx - (width / Decimal(2))
        y_max = cy + (height / Decimal(2))
        return (x_min + (Decimal(int(col)) / Decimal(max(1, W - 1))) * width,
                y_max - (Decimal(int(row)) / Decimal(max(1, H - 1))) * height)
