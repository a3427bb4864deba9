"""Perturbation-tier frames through the oracle, pass for pass.

TEST INFRASTRUCTURE ONLY (the oracle's frames and bench.py's CPU baseline / reference arm):
the frame driver of the reference's perturbation path restated around the C oracle
(ap_oracle.c), in the order the engine issues its passes -- reference orbit search
(ref_orbit.py), chained-BLA table, the render pass, histogram and colour, the SSAA edge
or resolve pass, and the Pauldelbrot rebase loop (math_core/engine.py:1718-2113 for the
CUDA path, :822-1046 for the CPU path) with its pixel selection restated below.

Only two parts reach into the engine's package, both outside the path bench.py times:
series-start coefficients (orders 4 and 8; ap_bbsa_coeffs, pinned bit for bit to the
reference's coefficients by tests/test_bbsa.py) and the Strict Metric fallback's
pixel inputs.  The ctypes structs of the C header (fractura_b200.abi) and the fixed
synthetic LUT (fractura_b200.palette) are data, not engine code.
"""
import math
from decimal import Decimal, localcontext

import numpy as np

import oracle
import ref_orbit
from fractura_b200 import abi
from fractura_b200.config import compute_floatexp_scale, decimal_context
from fractura_b200.palette import synthetic_lut

ONE_PASS = "One-Pass Rebasing"


def max_delta_c(ref_px, ref_py, w_sub, h_sub, dx, dy):
    """Largest |dc| over a w_sub x h_sub sub-sample grid for a reference at (ref_px, ref_py):
    the farthest corner, widened by 1e-6."""
    ex = max(abs(ref_px), abs(float(w_sub - 1) - ref_px)) * abs(dx)
    ey = max(abs(ref_py), abs(float(h_sub - 1) - ref_py)) * abs(dy)
    return float(np.hypot(ex, ey)) * (1.0 + 1e-6)


def select_rebase_pixel(glitch_map, iter_map, max_iter, visited, W, H):
    """Next reference pixel (row, col) of the rebase loop, or None
    (math_core/engine.py:853-912): glitched pixels binned on a 16 x 16 grid; in the
    most populated bin first the unvisited interior pixel nearest the bin's median,
    then the unvisited escaped pixel with the highest value, then the unvisited pixel
    nearest the median; failing every bin, the first unvisited glitched pixel."""
    gi = np.argwhere(glitch_map > 0)
    if len(gi) == 0:
        return None
    bins = np.clip((gi[:, 0] * 16) // H, 0, 15) * 16 + np.clip((gi[:, 1] * 16) // W, 0, 15)
    counts = np.bincount(bins, minlength=256)
    for b in np.argsort(-counts):
        if counts[b] == 0:
            break
        px = gi[bins == b]
        its = iter_map[px[:, 0], px[:, 1]]
        mr, mc = np.median(px[:, 0]), np.median(px[:, 1])
        inner = (its < 0) | (its >= max_iter)
        if np.any(inner):
            q = px[inner]
            for t in np.argsort((q[:, 0] - mr) ** 2 + (q[:, 1] - mc) ** 2):
                rc = (int(q[t, 0]), int(q[t, 1]))
                if rc not in visited:
                    return rc
        esc = (its > 0) & (its < max_iter)
        q = px[esc]
        for t in np.argsort(-its[esc]):
            rc = (int(q[t, 0]), int(q[t, 1]))
            if rc not in visited:
                return rc
        for t in np.argsort((px[:, 0] - mr) ** 2 + (px[:, 1] - mc) ** 2):
            rc = (int(px[t, 0]), int(px[t, 1]))
            if rc not in visited:
                return rc
    for t in range(len(gi)):
        rc = (int(gi[t, 0]), int(gi[t, 1]))
        if rc not in visited:
            return rc
    return None


class RebaseProgress:
    """When the rebase loop goes on (math_core/engine.py:835-848): glitches remain, more
    than the Strict Metric's limit in Strict mode, and the count fell within the last two
    passes."""

    def __init__(self, exhaustive, strict_limit):
        self.prev, self.stalls, self.passes = None, 0, 0
        self.exhaustive, self.strict_limit = exhaustive, strict_limit

    def go_on(self, n):
        if n == 0 or (self.exhaustive and n <= self.strict_limit):
            return False
        if self.prev is not None and n >= self.prev:
            self.stalls += 1
            if self.stalls >= 2:
                return False
        else:
            self.stalls = 0
        self.prev = n
        return True


def pert_frame(m, arith=abi.AP_ARITH_REF_CPU, lut=None, edge_threshold=0.35, max_passes=4,
                      bla_eps=None, fp32=False):
    """A perturbation-tier frame through the oracle, pass for pass as the engine issues it,
    including the rebase loop.  ``m`` is a view dict (W, H, factor, max_iter, cx, cy,
    width, scheme, fractal_type, julia_cx, julia_cy, gen_n, gen_kr, gen_ki, bbsa_order,
    glitch_mode; optional bbsa_tol, offset, density, contrast).  ``bla_eps`` selects the
    dc-aware BLA table (the engine's bla_form="accurate"); ``fp32`` the FP32-mantissa
    FloatExp form on the coarse passes (the engine's delta_form="fp32": pixel offsets in
    units of 2^-E with E from the view's width at every depth).  Returns (frame, rebase
    passes)."""
    W, H, f, mi = m["W"], m["H"], m["factor"], m["max_iter"]
    ft, scheme = m["fractal_type"], m["scheme"]
    cpu_sem = arith == abi.AP_ARITH_REF_CPU
    pw = Decimal(m["width"])
    cxd, cyd = Decimal(m["cx"]), Decimal(m["cy"])
    ctx = decimal_context(pw)
    floatexp = pw < Decimal("1e-300")
    e_scale = compute_floatexp_scale(pw) if floatexp else 0
    with localcontext(ctx):
        ph = pw * (Decimal(H) / Decimal(W))
        two_e = Decimal(2) ** e_scale
        dx_f = float(pw * two_e / Decimal(max(1, W - 1)))
        dy_f = float(ph * two_e / Decimal(max(1, H - 1)))
        fe_e = compute_floatexp_scale(pw)
        fe_dx = float(pw * (Decimal(2) ** fe_e) / Decimal(max(1, W - 1))) / float(f)
        fe_dy = float(ph * (Decimal(2) ** fe_e) / Decimal(max(1, H - 1))) / float(f)

    def coarse(q):
        """The params of a coarse pass: the FP32 form's, when selected."""
        if not fp32:
            return q
        c = abi.ApFrameParams.from_buffer_copy(q)
        c.tier = abi.AP_TIER_FLOATEXP32
        c.dx_hi, c.dy_hi, c.e_scale = fe_dx, fe_dy, int(fe_e)
        c.bbsa_skip = 0
        return c
    # the oracle's own Decimal restatement of the reference's orbit search (oracle/ref_orbit.py)
    bcx, bcy, bu, bv, re, im, rl = ref_orbit.find_reference(
        cxd, cyd, pw, ph, mi, ft=ft, julia_cx=m["julia_cx"], julia_cy=m["julia_cy"],
        n=m["gen_n"], kr=m["gen_kr"], ki=m["gen_ki"])
    order = m["bbsa_order"]
    if floatexp and order in (4, 8):
        order = 32  # the reference maps series starts to chained BLA on this tier
    max_r = float(pw) * 0.75
    inv_r = 1.0 / max_r if max_r > 0.0 else 1.0
    bbsa_tol = m.get("bbsa_tol", 1e-4)

    def series(r_re, r_im, r_len):
        if order not in (4, 8):
            return np.zeros(17, np.float64)  # no series start
        # series-start coefficients: the library's host function, pinned to the
        # reference's compute_bbsa_coeffs by tests/test_bbsa.py
        from fractura_b200 import _lib
        from fractura_b200.perturbation import bbsa_coefficients
        return bbsa_coefficients(_lib.load(), r_re, r_im, r_len, max_r, ft, bbsa_tol, order,
                                 m["gen_n"], m["gen_kr"], m["gen_ki"], e_scale)

    def set_series(q, c):
        q.bbsa_skip, q.bbsa_inv_r = int(c[0]), inv_r
        for t in range(16):
            q.bbsa[t] = float(c[1 + t])
    use_bla = order == 32 and ft in (0, 2, 4) and not (cpu_sem and scheme == 11)
    tol = 1e-6

    def table(r_re, r_im, r_len, rpx, rpy):
        if bla_eps is not None:
            dcm = math.ldexp(max_delta_c(rpx, rpy, W * f, H * f, dx_f / f, dy_f / f), -e_scale)
            return oracle.build_bla_dc(r_re, r_im, r_len, ft, bla_eps, dcm, 16, m["gen_n"], m["gen_kr"],
                                       m["gen_ki"])
        return oracle.build_bla(r_re, r_im, r_len, ft, tol, 16, m["gen_n"], m["gen_kr"], m["gen_ki"])

    fr = oracle.Frame(W, H, lut=synthetic_lut() if lut is None else lut)
    fr.ref_re, fr.ref_im = np.ascontiguousarray(re[:rl + 1]), np.ascontiguousarray(im[:rl + 1])
    fr.bla = table(re, im, rl, float(W - 1) * float(bu) * float(f),
                   float(H - 1) * float(bv) * float(f)) if use_bla else None
    one_pass = ONE_PASS in m["glitch_mode"]
    strict = 0 if one_pass else (1 if "Pauldelbrot" in m["glitch_mode"] or "Strict" in m["glitch_mode"] else 0)
    p = abi.new_params(width=W, height=H, factor=f, max_iter=mi, fractal_type=ft,
                       tier=abi.AP_TIER_FLOATEXP if floatexp else abi.AP_TIER_PERTURB, arith=arith,
                       e_scale=e_scale, gen_n=m["gen_n"], gen_kr=m["gen_kr"],
                       gen_ki=m["gen_ki"], scheme_id=scheme, num_bins=65536 if scheme == 11 else 2048,
                       dx_hi=dx_f / f, dy_hi=dy_f / f, ref_px=float(W - 1) * float(bu) * float(f),
                       ref_py=float(H - 1) * float(bv) * float(f), ref_cx=float(bcx), ref_cy=float(bcy),
                       julia_cx_hi=float(m["julia_cx"]), julia_cy_hi=float(m["julia_cy"]),
                       ref_len=int(rl), bla_levels=16 if use_bla else 0, strict_glitch=strict,
                       palette_offset=m.get("offset", 0.0), color_density=m.get("density", 1.0),
                       color_contrast=m.get("contrast", 1.0))
    set_series(p, series(re, im, rl))
    uf = (abi.AP_FLAG_ESCAPE_GLITCH | abi.AP_FLAG_NAN_GUARD) if cpu_sem else abi.AP_FLAG_NAN_GUARD
    rf = (abi.AP_FLAG_ESCAPE_GLITCH | abi.AP_FLAG_NAN_GUARD) if cpu_sem else abi.AP_FLAG_ESCAPE_GLITCH
    if one_pass:
        uf |= abi.AP_FLAG_REBASE
        rf |= abi.AP_FLAG_REBASE

    def resolve(q):
        bla_keep = fr.bla
        if not cpu_sem:
            fr.bla = None
            q.bla_levels = 0
        q.flags = rf
        oracle.resolve_hist_pass(q, fr)
        fr.bla = bla_keep

    if scheme == 11:
        p.flags = uf | abi.AP_FLAG_NO_RGB
        oracle.render_pass(coarse(p), fr)
        oracle.histogram_cdf(fr, mi)
        oracle.colour(p, fr)
        if f > 1:
            oracle.edge_detect(fr, np.float32(edge_threshold))
            q = abi.ApFrameParams.from_buffer_copy(p)
            resolve(q)
    else:
        p.flags = uf
        oracle.render_pass(coarse(p), fr)
        if f > 1:
            oracle.edge_detect(fr, np.float32(edge_threshold))
            p.mode = abi.AP_MODE_EDGE
            p.flags = uf | (0 if cpu_sem else abi.AP_FLAG_ITER_LAST_SUB)
            oracle.render_pass(p, fr)
    if not (strict and pw < Decimal("1e-12")):
        return fr, 0
    state = RebaseProgress("Strict" in m["glitch_mode"], 128 if cpu_sem else 512)
    visited = {(int(np.clip(p.ref_py / f, 0, H - 1)), int(np.clip(p.ref_px / f, 0, W - 1)))}
    bits = ref_orbit.prec_bits(pw)
    while state.passes < max_passes:
        g = fr.glitch_out.copy()
        if not state.go_on(int(np.count_nonzero(g))):
            break
        state.passes += 1
        chosen = select_rebase_pixel(g, fr.iter_map, mi, visited, W, H)
        if chosen is None:
            break
        visited.add(chosen)
        gr, gc = chosen
        r_cx, r_cy = ref_orbit.pixel_c(cxd, cyd, pw, ph, W, H, gc, gr)
        r_re, r_im, r_len = ref_orbit.orbit(r_cx, r_cy, mi, ft, m["julia_cx"], m["julia_cy"], bits,
                                            n=m["gen_n"], kr=m["gen_kr"], ki=m["gen_ki"])
        fr.ref_re, fr.ref_im = np.ascontiguousarray(r_re[:r_len + 1]), np.ascontiguousarray(r_im[:r_len + 1])
        fr.bla = table(r_re, r_im, r_len, float(gc) * f, float(gr) * f) if use_bla else None
        fr.glitch_in[...] = g
        q = abi.ApFrameParams.from_buffer_copy(p)
        q.ref_px, q.ref_py = float(gc) * f, float(gr) * f
        q.ref_cx, q.ref_cy = float(r_cx), float(r_cy)
        q.ref_len = int(r_len)
        q.bla_levels = 16 if use_bla else 0
        q.rebase_pass = state.passes
        set_series(q, series(r_re, r_im, r_len))
        if scheme == 11:
            resolve(q)
        elif f == 1:
            q.mode, q.flags = abi.AP_MODE_COARSE, uf
            oracle.render_pass(coarse(q), fr)
        elif cpu_sem:
            q.mode, q.flags = abi.AP_MODE_COARSE, uf
            oracle.render_pass(q, fr)
            q.mode = abi.AP_MODE_FULL
            oracle.render_pass(q, fr)
        else:
            q.mode, q.flags = abi.AP_MODE_FULL, uf | abi.AP_FLAG_ITER_LAST_SUB
            oracle.render_pass(q, fr)
    if "Strict" in m["glitch_mode"]:
        # every pixel still flagged: its own orbit, on the host in exact Decimal
        # arithmetic (CPU path; CUDA path beyond its device tiers) or in the CUDA
        # path's double-double / fixed-point tier
        from fractura_b200.perturbation import strict_device_inputs, strict_device_tier, strict_values
        coords = np.argwhere(fr.glitch_out > 0)
        tier = None if cpu_sem else strict_device_tier(pw, ft)
        if len(coords) and tier is None:
            vals = strict_values(coords, W, H, mi, cxd, cyd, pw, ph, ft, m["julia_cx"], m["julia_cy"],
                                 m["gen_n"], m["gen_kr"], m["gen_ki"], scalar=_decimal_escape)
            q = abi.ApFrameParams.from_buffer_copy(p)
            q.arith = abi.AP_ARITH_REF_CPU
            oracle.set_pixels(q, fr, coords, vals)
        elif len(coords):
            q, view, signs, limbs = strict_device_inputs(p, coords, tier, W, H, cxd, cyd, pw, ph, m["julia_cx"],
                                                         m["julia_cy"])
            oracle.strict_eval(q, fr, view, coords, signs, limbs)
    return fr, state.passes




def _decimal_escape(cx, cy, max_iter, fractal_type, julia_cx, julia_cy, bits, gen_n=3, gen_kr=0.25, gen_ki=1.0):
    """The Strict Metric's host value of one pixel, in Decimal (ref_orbit.escape)."""
    return ref_orbit.escape(cx, cy, max_iter, fractal_type, julia_cx, julia_cy, bits, n=gen_n, kr=gen_kr,
                            ki=gen_ki)
