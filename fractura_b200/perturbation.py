"""Perturbation tiers of render_frame: orbit, BLA table, passes and rebasing.

Host orchestration of math_core/engine.py:1807-2113 (FP64 deltas) and
:1718-1806 (FloatExp deltas): the reference orbit comes from
high_precision.find_optimal_reference_orbit (host, Decimal), is copied to
the device once per orbit, the chained-BLA table is built on the device
from it (ap_build_bla), and every pixel pass is one C-ABI launch.  The
Pauldelbrot rebase loop (math_core/engine.py:1890-2113) reads the glitch
and iteration maps back, picks a new reference pixel on the host
(select_rebase_pixel) and re-renders only the glitched pixels.
"""
import ctypes as C
import math
from decimal import Decimal, localcontext

import numpy as np

from . import abi, _lib
from .config import compute_floatexp_scale, compute_required_prec_bits, decimal_context
from . import high_precision as hp

BLA_LEVELS = 16
MAX_REBASE_PASSES = 4
# glitch_mode of the one-pass rebasing form (AP_FLAG_REBASE): every pixel restarts its
# delta from the orbit's start when |z| < |dz| or the reference ends, in the same pass.
# The reference has no such mode; its modes re-render glitched pixels around new references.
ONE_PASS_REBASING = "One-Pass Rebasing"

# Host<->device traffic of the last perturbation frame (bytes), for benchmarking.
LAST_FRAME_STATS = {"h2d_bytes": 0, "d2h_bytes": 0, "rebase_passes": 0, "strict_pixels": 0, "strict_tier": 0}


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _pick_in_cluster(cluster, its, max_iter, visited):
    """The reference's choice inside one grid cell (math_core/engine.py:1943-1985):
    cluster = glitched (row, col) in row-major order, its = their smooth values."""
    cr = np.median(cluster[:, 0])
    cc = np.median(cluster[:, 1])
    interior = (its < 0) | (its >= max_iter)
    if np.any(interior):
        pts = cluster[interior]
        dists = (pts[:, 0] - cr) ** 2 + (pts[:, 1] - cc) ** 2
        for d in np.argsort(dists):
            cand = (int(pts[d, 0]), int(pts[d, 1]))
            if cand not in visited:
                return cand
    escaped = (its > 0) & (its < max_iter)
    cands = cluster[escaped]
    if len(cands) > 0:
        for c in np.argsort(-its[escaped]):
            cand = (int(cands[c, 0]), int(cands[c, 1]))
            if cand not in visited:
                return cand
    dists = (cluster[:, 0] - cr) ** 2 + (cluster[:, 1] - cc) ** 2
    for d in np.argsort(dists):
        cand = (int(cluster[d, 0]), int(cluster[d, 1]))
        if cand not in visited:
            return cand
    return None


def select_rebase_pixel(glitch_map, iter_map, max_iter, visited, W, H):
    """Next reference pixel (row, col) for a rebase pass, or None.

    Bins glitched pixels on a 16x16 grid; in the most populated bin first an
    unvisited interior pixel closest to the bin's median, then the unvisited
    escaped pixel with the highest smooth value, then the unvisited pixel
    closest to the median; failing every bin, the first unvisited glitched
    pixel (math_core/engine.py:1923-1992).
    """
    gi = np.argwhere(glitch_map > 0)
    if len(gi) == 0:
        return None
    bin_r = np.clip((gi[:, 0] * 16) // H, 0, 15)
    bin_c = np.clip((gi[:, 1] * 16) // W, 0, 15)
    bin_idx = bin_r * 16 + bin_c
    counts = np.bincount(bin_idx, minlength=256)
    for b in np.argsort(-counts):
        if counts[b] == 0:
            break
        cluster = gi[bin_idx == b]
        cand = _pick_in_cluster(cluster, iter_map[cluster[:, 0], cluster[:, 1]], max_iter, visited)
        if cand is not None:
            return cand
    for g in range(len(gi)):
        cand = (int(gi[g, 0]), int(gi[g, 1]))
        if cand not in visited:
            return cand
    return None


def _cell_spans(n):
    """[start, stop) of the pixels whose cell index min(15, 16 p // n) is 0..15."""
    cell = np.minimum((np.arange(n) * 16) // n, 15)
    return [(int(np.searchsorted(cell, q, "left")), int(np.searchsorted(cell, q, "right")))
            for q in range(16)]


def select_rebase_pixel_binned(counts, fetch_cell, fetch_all, max_iter, visited, W, H):
    """select_rebase_pixel from the grid's cell counts (ap_glitch_bins): only the
    cells it inspects are fetched (fetch_cell(r0, r1, c0, c1) -> glitch and smooth
    values of that rectangle), the whole maps only when every cell is exhausted
    (fetch_all()).  Same result as select_rebase_pixel on the whole maps: a cell's
    glitched pixels in row-major order are the whole map's, restricted to the cell."""
    counts = np.asarray(counts, dtype=np.int64)
    if counts.sum() == 0:
        return None
    rows, cols = _cell_spans(H), _cell_spans(W)
    for b in np.argsort(-counts):
        if counts[b] == 0:
            break
        (r0, r1), (c0, c1) = rows[b // 16], cols[b % 16]
        g, it = fetch_cell(r0, r1, c0, c1)
        loc = np.argwhere(g > 0)
        cluster = loc + np.array([r0, c0])
        cand = _pick_in_cluster(cluster, it[loc[:, 0], loc[:, 1]], max_iter, visited)
        if cand is not None:
            return cand
    g, _ = fetch_all()
    gi = np.argwhere(g > 0)
    for q in range(len(gi)):
        cand = (int(gi[q, 0]), int(gi[q, 1]))
        if cand not in visited:
            return cand
    return None


class RebaseState:
    """Progress bookkeeping of the rebase loop (math_core/engine.py:1893-1919)."""

    def __init__(self, init_rc, exhaustive, strict_limit=512):
        self.visited = {init_rc}
        self.prev = None
        self.no_progress = 0
        self.passes = 0
        self.exhaustive = exhaustive
        self.strict_limit = strict_limit

    def should_continue(self, n_glitched):
        if n_glitched == 0:
            return False
        if self.exhaustive and n_glitched <= self.strict_limit:
            return False
        if self.prev is not None and n_glitched >= self.prev:
            self.no_progress += 1
            if self.no_progress >= 2:
                return False
        else:
            self.no_progress = 0
        self.prev = n_glitched
        return True


def _upload_orbit(torch, re, im, ref_len, slot, tag):
    from .engine import get_scratch_device_array_1d
    n = ref_len + 1
    d_re = get_scratch_device_array_1d(n, np.float64, f"{tag}_re_{slot}")[:n]
    d_im = get_scratch_device_array_1d(n, np.float64, f"{tag}_im_{slot}")[:n]
    d_re.copy_(torch.from_numpy(np.ascontiguousarray(re[:n])), non_blocking=False)
    d_im.copy_(torch.from_numpy(np.ascontiguousarray(im[:n])), non_blocking=False)
    LAST_FRAME_STATS["h2d_bytes"] += 16 * n
    return d_re, d_im


def _build_bla(L, d_re, d_im, ref_len, fractal_type, tol, gen_n, gen_kr, gen_ki, slot, stream_h,
               tag="ref", eps=None, dc_max=None):
    """The chained-BLA table of one reference orbit: the reference's merge at
    ``tol``, or with ``eps`` the dc-aware merge for deltas up to ``dc_max``."""
    from .engine import get_scratch_device_array_1d
    n = BLA_LEVELS * max(ref_len, 1) * 5
    table = get_scratch_device_array_1d(n, np.float64, f"bla_table_{tag}_{slot}")[:n]
    if eps is None:
        _lib.launch(L.ap_build_bla, _ptr(d_re), _ptr(d_im), int(ref_len), int(fractal_type),
                    float(tol), BLA_LEVELS, int(gen_n), float(gen_kr), float(gen_ki),
                    _ptr(table), stream_h, what="ap_build_bla")
    else:
        _lib.launch(L.ap_build_bla_dc, _ptr(d_re), _ptr(d_im), int(ref_len), int(fractal_type),
                    float(eps), float(dc_max), BLA_LEVELS, int(gen_n), float(gen_kr), float(gen_ki),
                    _ptr(table), stream_h, what="ap_build_bla_dc")
    return table


def bbsa_coefficients(L, re, im, ref_len, max_r, fractal_type, tol, order, gen_n, gen_kr, gen_ki,
                      e_scale):
    """(skip, a1_re, a1_im, ..., a8_re, a8_im) of the series start for one reference orbit
    (ap_bbsa_coeffs, host code of the library; compute_bbsa_coeffs,
    math_core/high_precision.py:537)."""
    out = np.zeros(17, np.float64)
    r = np.ascontiguousarray(re[:max(ref_len, 1) + 1], np.float64)
    i = np.ascontiguousarray(im[:max(ref_len, 1) + 1], np.float64)
    _lib.check(L.ap_bbsa_coeffs(r.ctypes.data_as(C.c_void_p), i.ctypes.data_as(C.c_void_p),
                                int(ref_len), float(max_r), int(fractal_type), float(tol), int(order),
                                int(gen_n), float(gen_kr), float(gen_ki), int(e_scale),
                                out.ctypes.data_as(C.c_void_p)), "ap_bbsa_coeffs")
    return out


def _set_series(p, series, inv_r):
    p.bbsa_skip = int(series[0])
    p.bbsa_inv_r = float(inv_r)
    for q in range(16):
        p.bbsa[q] = float(series[1 + q])


def max_delta_c(ref_px, ref_py, w_sub, h_sub, dx, dy):
    """Largest |dc| over a w_sub x h_sub sub-sample grid for a reference at
    sub-sample (ref_px, ref_py): the farthest corner, widened by 1e-6 so that
    rounding of the per-pixel deltas stays inside."""
    ex = max(abs(ref_px), abs(float(w_sub - 1) - ref_px)) * abs(dx)
    ey = max(abs(ref_py), abs(float(h_sub - 1) - ref_py)) * abs(dy)
    return float(np.hypot(ex, ey)) * (1.0 + 1e-6)


def _pack_orbit(L, d_re, d_im, ref_len, slot, tag, stream_h):
    from .engine import get_scratch_device_array_1d
    n = 6 * (ref_len + 1)  # FP64 records, then the FP32 copy of the FP32 FloatExp tier
    packed = get_scratch_device_array_1d(n, np.float64, f"{tag}_orbit_packed_{slot}")[:n]
    _lib.launch(L.ap_pack_orbit, _ptr(d_re), _ptr(d_im), int(ref_len), _ptr(packed), stream_h,
                what="ap_pack_orbit")
    return packed


def _pack_bla(L, table, ref_len, slot, tag, stream_h, orbit_packed):
    """Packed BLA rows; also fills the level-0 radius of the packed orbit records."""
    from .engine import get_scratch_device_array_1d
    n = 80 * max(ref_len, 1)
    packed = get_scratch_device_array_1d(n, np.float64, f"bla_packed_{tag}_{slot}")[:n]
    _lib.launch(L.ap_pack_bla, _ptr(table), BLA_LEVELS, int(ref_len), _ptr(packed), _ptr(orbit_packed),
                stream_h, what="ap_pack_bla")
    return packed


def _inputs(L, d_re, d_im, ref_len, bla, slot, tag, stream_h, fp32=False):
    """Packed orbit (always), packed BLA table (when leaps are used) and, for the
    FP32 FloatExp tier, the FP32 orbit copy and BLA records."""
    from .engine import get_scratch_device_array_1d
    po = _pack_orbit(L, d_re, d_im, ref_len, slot, tag, stream_h)
    pb = _pack_bla(L, bla, ref_len, slot, tag, stream_h, po) if (bla is not None and ref_len > 0) else None
    pf = None
    if fp32:
        n4 = 4 * (ref_len + 1)
        if bla is not None and ref_len > 0:
            nb = 80 * ref_len
            pf = get_scratch_device_array_1d(nb, np.float64, f"bla_fe32_{tag}_{slot}")[:nb]
        _lib.launch(L.ap_pack_fe32, _ptr(po), int(ref_len), _ptr(bla) if pf is not None else None,
                    BLA_LEVELS, _ptr(po[n4:]), _ptr(pf), stream_h, what="ap_pack_fe32")
    return po, pb, pf


def _with_packed(b, packed, fp32=False):
    b.orbit_packed = _ptr(packed[0])
    b.bla_packed = _ptr(packed[2] if fp32 else packed[1])
    return b


def _coarse_params(p, fe32):
    """Params of a coarse pass: the FP32 FloatExp tier in normalised units when enabled."""
    if fe32 is None:
        return p
    q = _copy_params(p)
    q.tier = abi.AP_TIER_FLOATEXP32
    q.dx_hi, q.dy_hi, q.e_scale = fe32
    q.bbsa_skip = 0
    return q


def probe_perturbation_params(p, *, W, H, search_max, center_x_dec, center_y_dec, plot_width_dec,
                              tier, fractal_type, julia_cx, julia_cy, bbsa_tol, bbsa_order, gen_n,
                              gen_kr, gen_ki, arith_code):
    """Reference orbit and parameters of the adaptive max-iter probe's perturbation
    branches (math_core/engine.py:1120-1179 on the CPU, :1212-1278 on the device).

    Unlike a frame: the series start keeps ``bbsa_tol`` / ``bbsa_order`` as given on
    the FloatExp tier too, with its radius 0.75 w in 2^-E units there; no chained-BLA
    leaps; no glitch test (strict_glitch 0).  The sample variant is the plain one: the
    CPU kernels flag escape glitches and guard NaN, the device's plain sample
    (math_core/cuda_kernels.py:422, :819) flags escape glitches only.  Returns the host
    orbit (re, im, ref_len); ``p`` is filled for one coarse pass at factor 1."""
    ctx = decimal_context(plot_width_dec)
    floatexp = tier == abi.AP_TIER_FLOATEXP
    with localcontext(ctx):
        plot_height_dec = plot_width_dec * (Decimal(H) / Decimal(W))
        e_scale = compute_floatexp_scale(plot_width_dec) if floatexp else 0
        scale = Decimal(2) ** e_scale
        w_view = plot_width_dec * scale
        dx_f = float(w_view / Decimal(max(1, W - 1)))
        dy_f = float(plot_height_dec * scale / Decimal(max(1, H - 1)))
    bcx, bcy, bu, bv, re, im, ref_len = hp.find_optimal_reference_orbit(
        center_x_dec, center_y_dec, plot_width_dec, plot_height_dec, search_max, W, H,
        fractal_type=fractal_type, julia_cx=julia_cx, julia_cy=julia_cy, gen_n=gen_n,
        gen_kr=gen_kr, gen_ki=gen_ki, is_floatexp=floatexp)
    max_r = float(w_view) * 0.75
    series = bbsa_coefficients(_lib.load(), re, im, ref_len, max_r, fractal_type, bbsa_tol, bbsa_order,
                               gen_n, gen_kr, gen_ki, e_scale)
    _set_series(p, series, 1.0 / max_r if max_r > 0.0 else 1.0)
    p.dx_hi, p.dy_hi = dx_f, dy_f
    p.ref_px = float(W - 1) * float(bu)
    p.ref_py = float(H - 1) * float(bv)
    p.ref_cx, p.ref_cy = float(bcx), float(bcy)
    p.julia_cx_hi, p.julia_cy_hi = float(julia_cx), float(julia_cy)
    p.ref_len = int(ref_len)
    p.e_scale = int(e_scale)
    p.bla_levels = 0
    p.strict_glitch = 0
    p.rebase_pass = 0
    p.mode = abi.AP_MODE_COARSE
    cpu_sem = arith_code == abi.AP_ARITH_REF_CPU
    p.flags = abi.AP_FLAG_NO_RGB | abi.AP_FLAG_ESCAPE_GLITCH | (abi.AP_FLAG_NAN_GUARD if cpu_sem else 0)
    return re, im, ref_len


def render_perturbation_frame(p, fr, lut, stream_h, st, *, W, H, factor, max_iter, center_x_dec,
                              center_y_dec, plot_width_dec, tier, scheme, num_bins, fractal_type,
                              julia_cx, julia_cy, bbsa_tol, bbsa_order, glitch_mode, gen_n, gen_kr,
                              gen_ki, edge_threshold, slot, arith_code, extra_out=None,
                              fp32_deltas=False, bla_eps=None, rows=None, orbit=None):
    """All device passes of one perturbation-tier frame (math_core/engine.py:1718-2113).

    ``orbit`` (ref_cx, ref_cy, u, v, re, im, ref_len) replaces the reference search (a
    split frame's ranks share rank 0's).  ``rows`` = (r0, r1) renders only that band of
    the coarse pass (ap_render_rows) into the frame-size buffers and returns: no colour,
    histogram or rebase pass (the split frame does those across ranks); it serves
    factor 1 and the glitch modes that need no re-render pass."""
    import torch
    from .engine import _buffers, get_scratch_device_array
    L = _lib.load()
    cpu_sem = arith_code == abi.AP_ARITH_REF_CPU
    kmap = s64 = None
    if extra_out is not None:
        kmap, s64 = extra_out
    ctx = decimal_context(plot_width_dec)
    with localcontext(ctx):
        plot_height_dec = plot_width_dec * (Decimal(H) / Decimal(W))
        dx_f = float(plot_width_dec / Decimal(max(1, W - 1)))
        dy_f = float(plot_height_dec / Decimal(max(1, H - 1)))
        floatexp = tier == abi.AP_TIER_FLOATEXP
        if floatexp:
            e_scale = compute_floatexp_scale(plot_width_dec)
            norm_w = plot_width_dec * (Decimal(2) ** e_scale)
            norm_h = plot_height_dec * (Decimal(2) ** e_scale)
            dx_f = float(norm_w / Decimal(max(1, W - 1)))
            dy_f = float(norm_h / Decimal(max(1, H - 1)))
            if bbsa_order in (4, 8):
                bbsa_order = 32
                if bbsa_tol > 1e-6:
                    bbsa_tol = 1e-6
        else:
            e_scale = 0
        # FP32 FloatExp tier: the same spacing in units of 2^-E (E from config.py:51).
        fe32 = None
        if fp32_deltas:
            fe_e = compute_floatexp_scale(plot_width_dec)
            fe32 = (float(plot_width_dec * (Decimal(2) ** fe_e) / Decimal(max(1, W - 1))) / float(factor),
                    float(plot_height_dec * (Decimal(2) ** fe_e) / Decimal(max(1, H - 1))) / float(factor),
                    int(fe_e))
    one_pass = ONE_PASS_REBASING in glitch_mode
    if arith_code == abi.AP_ARITH_FAST and not one_pass:
        raise ValueError(f"arith='fast' serves glitch_mode {ONE_PASS_REBASING!r} only")
    # the FP32 form rebases at every depth; below 1e-300 its SSAA edge pass would need
    # FP64 FloatExp rebasing, which is not built
    if one_pass and (fractal_type in (2, 3) or (tier != abi.AP_TIER_PERTURB and (not fp32_deltas or factor > 1))):
        raise NotImplementedError(
            f"{ONE_PASS_REBASING!r} serves Mandelbrot, Burning Ship and Multibrot frames: FP64 deltas "
            "(widths 1e-300 .. 1e-12), or delta_form='fp32' (any depth; factor 1 below 1e-300)")
    strict = 0 if one_pass else (1 if ("Auto Rebasing" in glitch_mode or "Strict" in glitch_mode
                                       or "Pauldelbrot" in glitch_mode) else 0)
    LAST_FRAME_STATS.update(h2d_bytes=0, d2h_bytes=0, rebase_passes=0, strict_pixels=0, strict_tier=0)

    if rows is not None and (factor != 1 or strict):
        raise NotImplementedError("a band of a frame serves factor 1 with glitch modes 'One-Pass Rebasing' "
                                  "or 'Off (Single-Ref)'")
    if orbit is None:
        orbit = hp.find_optimal_reference_orbit(
            center_x_dec, center_y_dec, plot_width_dec, plot_height_dec, max_iter, W, H,
            fractal_type=fractal_type, julia_cx=julia_cx, julia_cy=julia_cy, gen_n=gen_n,
            gen_kr=gen_kr, gen_ki=gen_ki, is_floatexp=floatexp)
    bcx, bcy, bu, bv, re, im, ref_len = orbit
    # Series-approximation start (math_core/engine.py:1816-1840): radius 0.75 w, same
    # inverse radius for every reference of the frame.
    max_r = float(plot_width_dec) * 0.75
    bbsa_inv_r = 1.0 / max_r if max_r > 0.0 else 1.0
    series = bbsa_coefficients(L, re, im, ref_len, max_r, fractal_type, bbsa_tol, bbsa_order,
                               gen_n, gen_kr, gen_ki, e_scale)
    d_re, d_im = _upload_orbit(torch, re, im, ref_len, slot, "ref")
    # The CPU reference's histogram path evaluates samples without BLA leaps
    # (math_core/engine.py:624-637, cpu_kernels.py:1887); every other path leaps.
    use_bla = bbsa_order == 32 and fractal_type in (0, 2, 4) and not (cpu_sem and scheme == 11)
    p.dx_hi, p.dy_hi = dx_f / float(factor), dy_f / float(factor)
    p.ref_px = float(W - 1) * float(bu) * float(factor)
    p.ref_py = float(H - 1) * float(bv) * float(factor)
    ws, hs = W * factor, H * factor
    # |dc|max of the dc-aware table in absolute units (the FloatExp tier's spacing is in 2^-E units)
    def dc_max_at(rpx, rpy):
        return math.ldexp(max_delta_c(rpx, rpy, ws, hs, p.dx_hi, p.dy_hi), -int(e_scale))

    bla = _build_bla(L, d_re, d_im, ref_len, fractal_type, bbsa_tol, gen_n, gen_kr, gen_ki,
                     slot, stream_h, eps=bla_eps,
                     dc_max=dc_max_at(p.ref_px, p.ref_py)) if use_bla else None
    packed = _inputs(L, d_re, d_im, ref_len, bla, slot, "ref", stream_h, fp32=fe32 is not None)

    p.ref_cx, p.ref_cy = float(bcx), float(bcy)
    p.julia_cx_hi, p.julia_cy_hi = float(julia_cx), float(julia_cy)
    p.ref_len = int(ref_len)
    p.e_scale = int(e_scale)
    p.strict_glitch = strict
    p.bla_levels = BLA_LEVELS if use_bla else 0
    _set_series(p, series, bbsa_inv_r)
    p.rebase_pass = 0
    # Sample variant: the CPU reference flags both; the CUDA unified kernels use the
    # BLA variant (NaN guard), their histogram resolve passes the plain one (escape glitch).
    unified_flags = (abi.AP_FLAG_ESCAPE_GLITCH | abi.AP_FLAG_NAN_GUARD) if cpu_sem else abi.AP_FLAG_NAN_GUARD
    resolve_flags = (abi.AP_FLAG_ESCAPE_GLITCH | abi.AP_FLAG_NAN_GUARD) if cpu_sem else abi.AP_FLAG_ESCAPE_GLITCH
    if one_pass:
        unified_flags |= abi.AP_FLAG_REBASE
        resolve_flags |= abi.AP_FLAG_REBASE
    _lib.device_op(fr.glitch_in.zero_)
    orbit = (d_re, d_im)
    cdf = None
    if rows is not None:
        p.mode = abi.AP_MODE_COARSE
        p.flags = unified_flags | abi.AP_FLAG_NO_RGB
        b = _with_packed(_buffers(fr, lut, orbit=orbit, bla=bla, kmap=kmap, s64=s64), packed, fe32 is not None)
        q = _coarse_params(p, fe32)
        r0, r1 = int(rows[0]), int(rows[1])
        _lib.launch(L.ap_render_rows, C.byref(q), C.byref(b), r0, r1 - r0, stream_h, what="ap_render_rows")
        return dict(ref_len=ref_len, passes=0)

    if scheme == 11:
        hist = get_scratch_device_array((num_bins,), np.int32, f"hist_bins_{slot}")
        cdf = get_scratch_device_array((num_bins,), np.float32, f"cdf_lut_{slot}")
        p.mode = abi.AP_MODE_COARSE
        p.flags = unified_flags | abi.AP_FLAG_NO_RGB
        b = _with_packed(_buffers(fr, lut, cdf=cdf, orbit=orbit, bla=bla, kmap=kmap, s64=s64), packed,
                         fe32 is not None)
        q = _coarse_params(p, fe32)
        _lib.launch(L.ap_render_pass, C.byref(q), C.byref(b), stream_h, what="ap_render_pass")
        _lib.launch(L.ap_histogram_cdf, _ptr(fr.iter), W, H, max_iter, num_bins, _ptr(hist), _ptr(cdf),
                                      stream_h, what="ap_histogram_cdf")
        _lib.launch(L.ap_colour, C.byref(p), C.byref(b), stream_h, what="ap_colour")
        if factor > 1:
            fr.edge_mask()
            _lib.launch(L.ap_edge_detect, _ptr(fr.iter), _ptr(fr.edge), W, H,
                                        float(np.float32(edge_threshold)), stream_h, what="ap_edge_detect")
            q = _resolve_params(p, resolve_flags, cpu_sem)
            b = _buffers(fr, lut, cdf=cdf, orbit=orbit, bla=bla if cpu_sem else None)
            _lib.launch(L.ap_resolve_hist_pass, C.byref(q), C.byref(b), stream_h, what="ap_resolve_hist_pass")
    else:
        p.mode = abi.AP_MODE_COARSE
        p.flags = unified_flags | abi.AP_FLAG_NO_RGB
        b = _with_packed(_buffers(fr, lut, orbit=orbit, bla=bla, kmap=kmap, s64=s64), packed,
                         fe32 is not None)
        q = _coarse_params(p, fe32)
        _lib.launch(L.ap_render_pass, C.byref(q), C.byref(b), stream_h, what="ap_render_pass")
        _lib.launch(L.ap_colour, C.byref(p), C.byref(b), stream_h, what="ap_colour")
        p.flags = unified_flags
        if factor > 1:
            fr.edge_mask()
            _lib.launch(L.ap_edge_detect, _ptr(fr.iter), _ptr(fr.edge), W, H,
                                        float(np.float32(edge_threshold)), stream_h, what="ap_edge_detect")
            p.mode = abi.AP_MODE_EDGE
            p.flags = unified_flags | (0 if cpu_sem else abi.AP_FLAG_ITER_LAST_SUB)
            b = _buffers(fr, lut, orbit=orbit, bla=bla)
            _lib.launch(L.ap_render_pass, C.byref(p), C.byref(b), stream_h, what="ap_render_pass")

    allow = strict == 1
    if not (allow and plot_width_dec < Decimal("1e-12")):
        return dict(ref_len=ref_len, passes=0)

    exhaustive = "Strict" in glitch_mode
    state = RebaseState((int(np.clip(p.ref_py / factor, 0, H - 1)), int(np.clip(p.ref_px / factor, 0, W - 1))),
                        exhaustive, strict_limit=128 if cpu_sem else 512)
    bits = compute_required_prec_bits(plot_width_dec)
    d_counts = torch.empty(256, dtype=torch.int32, device=fr.glitch_out.device)

    def fetch_cell(r0, r1, c0, c1):
        g = fr.glitch_out[r0:r1, c0:c1].cpu().numpy()
        it = fr.iter[r0:r1, c0:c1].cpu().numpy()
        LAST_FRAME_STATS["d2h_bytes"] += g.nbytes + it.nbytes
        return g, it

    def fetch_all():
        return fetch_cell(0, H, 0, W)

    while state.passes < MAX_REBASE_PASSES:
        # the glitch map's 16 x 16 cell counts come from the device (1 KB), then
        # only the cells the choice inspects
        _lib.launch(L.ap_glitch_bins, _ptr(fr.glitch_out), W, H, _ptr(d_counts), stream_h,
                    what="ap_glitch_bins")
        st.synchronize()
        counts = d_counts.cpu().numpy().astype(np.int64)
        LAST_FRAME_STATS["d2h_bytes"] += counts.size * 4
        n_gl = int(counts.sum())
        if not state.should_continue(n_gl):
            break
        state.passes += 1
        LAST_FRAME_STATS["rebase_passes"] = state.passes
        chosen = select_rebase_pixel_binned(counts, fetch_cell, fetch_all, max_iter, state.visited, W, H)
        if chosen is None:
            break
        g_row, g_col = chosen
        state.visited.add(chosen)
        with localcontext(ctx):
            x_min_dec = center_x_dec - (plot_width_dec / Decimal(2))
            y_max_dec = center_y_dec + (plot_height_dec / Decimal(2))
            r_cx = x_min_dec + (Decimal(int(g_col)) / Decimal(max(1, W - 1))) * plot_width_dec
            r_cy = y_max_dec - (Decimal(int(g_row)) / Decimal(max(1, H - 1))) * plot_height_dec
        r_re, r_im, r_len = hp.compute_single_highprec_orbit(
            r_cx, r_cy, max_iter, fractal_type, julia_cx, julia_cy, bits,
            gen_n=gen_n, gen_kr=gen_kr, gen_ki=gen_ki)
        if r_len > 100:
            hp.cache_reference_orbit(r_cx, r_cy, plot_width_dec, max_iter, r_re, r_im, r_len,
                                     fractal_type=fractal_type, julia_cx=julia_cx,
                                     julia_cy=julia_cy, gen_n=gen_n, gen_kr=gen_kr,
                                     gen_ki=gen_ki, is_floatexp=floatexp)
        # Each pass keeps its own orbit and table, so a recorded frame can be replayed.
        tag = f"rebase{state.passes}"
        d_re, d_im = _upload_orbit(torch, r_re, r_im, r_len, slot, tag)
        _lib.device_op(lambda: fr.glitch_in.copy_(fr.glitch_out))
        bla = _build_bla(L, d_re, d_im, r_len, fractal_type, bbsa_tol, gen_n, gen_kr, gen_ki,
                         slot, stream_h, tag, eps=bla_eps,
                         dc_max=dc_max_at(float(g_col) * factor, float(g_row) * factor)) if use_bla else None
        packed = _inputs(L, d_re, d_im, r_len, bla, slot, tag, stream_h, fp32=fe32 is not None)
        q = _copy_params(p)
        q.ref_px, q.ref_py = float(g_col) * float(factor), float(g_row) * float(factor)
        q.ref_cx, q.ref_cy = float(r_cx), float(r_cy)
        q.ref_len = int(r_len)
        q.bla_levels = BLA_LEVELS if bla is not None else 0
        q.rebase_pass = state.passes
        _set_series(q, bbsa_coefficients(L, r_re, r_im, r_len, max_r, fractal_type, bbsa_tol,
                                         bbsa_order, gen_n, gen_kr, gen_ki, e_scale), bbsa_inv_r)
        orbit = (d_re, d_im)
        if scheme == 11 and cdf is not None:
            q = _resolve_params(q, resolve_flags, cpu_sem)
            b = _buffers(fr, lut, cdf=cdf, orbit=orbit, bla=bla if cpu_sem else None, kmap=kmap, s64=s64)
            _lib.launch(L.ap_resolve_hist_pass, C.byref(q), C.byref(b), stream_h, what="ap_resolve_hist_pass")
        elif factor == 1:
            q.mode = abi.AP_MODE_COARSE
            q.flags = unified_flags | abi.AP_FLAG_NO_RGB
            b = _with_packed(_buffers(fr, lut, orbit=orbit, bla=bla, kmap=kmap, s64=s64), packed,
                             fe32 is not None)
            qc = _coarse_params(q, fe32)
            _lib.launch(L.ap_render_pass, C.byref(qc), C.byref(b), stream_h, what="ap_render_pass")
            _lib.launch(L.ap_colour, C.byref(q), C.byref(b), stream_h, what="ap_colour")
        else:
            b = _buffers(fr, lut, orbit=orbit, bla=bla, kmap=kmap, s64=s64)
            if cpu_sem:
                # CPU reference: coarse re-render of glitched pixels, then their supersample.
                q.mode = abi.AP_MODE_COARSE
                q.flags = unified_flags | abi.AP_FLAG_NO_RGB
                b = _with_packed(b, packed)
                _lib.launch(L.ap_render_pass, C.byref(q), C.byref(b), stream_h, what="ap_render_pass")
                q.flags = unified_flags
                q.mode = abi.AP_MODE_FULL
                b = _buffers(fr, lut, orbit=orbit, bla=bla)
            else:
                q.mode = abi.AP_MODE_FULL
                q.flags = unified_flags | abi.AP_FLAG_ITER_LAST_SUB
            _lib.launch(L.ap_render_pass, C.byref(q), C.byref(b), stream_h, what="ap_render_pass")
    if exhaustive:
        st.synchronize()
        g_all = fr.glitch_out.cpu().numpy()
        LAST_FRAME_STATS["d2h_bytes"] += g_all.nbytes
        coords = np.argwhere(g_all > 0)
        if len(coords):
            dev = fr.iter.device

            def upload(a):
                t = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
                LAST_FRAME_STATS["h2d_bytes"] += t.numel() * t.element_size()
                return t

            d_coords = upload(coords.astype(np.int32))
            b = _buffers(fr, lut, cdf=cdf if scheme == 11 else None)
            tier = None if cpu_sem else strict_device_tier(plot_width_dec, fractal_type)
            LAST_FRAME_STATS.update(strict_pixels=int(len(coords)), strict_tier=int(tier or 0))
            if tier is None:
                # host evaluation (the CPU path, and the CUDA path beyond its device
                # tiers), coloured with the CPU transfer functions
                values = strict_values(coords, W, H, max_iter, center_x_dec, center_y_dec, plot_width_dec,
                                       plot_height_dec, fractal_type, julia_cx, julia_cy, gen_n, gen_kr,
                                       gen_ki)
                d_vals = upload(values)
                q = _copy_params(p)
                q.arith = abi.AP_ARITH_REF_CPU
                _lib.launch(L.ap_set_pixels, C.byref(q), C.byref(b), _ptr(d_coords), _ptr(d_vals),
                            int(len(coords)), stream_h, what="ap_set_pixels")
            else:
                q, view, signs, limbs = strict_device_inputs(p, coords, tier, W, H, center_x_dec, center_y_dec,
                                                             plot_width_dec, plot_height_dec, julia_cx,
                                                             julia_cy)
                d_signs = upload(signs) if signs is not None else None
                d_limbs = upload(limbs.view(np.int32)) if limbs is not None else None
                _lib.launch(L.ap_strict_eval, C.byref(q), C.byref(b), C.byref(view), _ptr(d_coords),
                            _ptr(d_signs), _ptr(d_limbs), int(len(coords)), stream_h, what="ap_strict_eval")
            st.synchronize()
    return dict(ref_len=ref_len, passes=state.passes)


def strict_device_tier(plot_width_dec, fractal_type):
    """Device tier of the CUDA path's Strict Metric fallback (math_core/engine.py:285-296,
    :330): FP64 down to 1e-12, double-double down to 1e-30, 34-limb fixed point down to
    1e-315 except for Multibrot, None where the reference evaluates on the host."""
    if plot_width_dec >= Decimal("1e-12"):
        return abi.AP_STRICT_FP64
    if plot_width_dec >= Decimal("1e-30"):
        return abi.AP_STRICT_DD
    if plot_width_dec >= Decimal("1e-315") and fractal_type != 4:
        return abi.AP_STRICT_LIMBS
    return None


def fixed_limbs(d):
    """(sign, 34 uint32 limbs) of a Decimal: limb 0 the integer part, then 33 fraction
    limbs of floor(|d| 2^1056), most significant first (decimal_to_limbs,
    math_core/cuda_kernels.py:2242-2274, whose Decimal steps run at 500+ digits and so
    reproduce the exact floor)."""
    sign = 1 if d < 0 else 0
    t = d.copy_abs().as_tuple()  # exact: abs() would round to the context
    coeff = int("".join(map(str, t.digits))) if t.digits else 0
    frac_bits = 32 * (abi.AP_STRICT_NLIMBS - 1)
    if t.exponent >= 0:
        f = (coeff * 10 ** t.exponent) << frac_bits
    else:
        f = (coeff << frac_bits) // (10 ** (-t.exponent))
    f &= (1 << (32 * abi.AP_STRICT_NLIMBS)) - 1
    return sign, np.frombuffer(f.to_bytes(4 * abi.AP_STRICT_NLIMBS, "big"), dtype=">u4").astype(np.uint32)


def strict_device_inputs(p, coords, tier, W, H, center_x_dec, center_y_dec, plot_width_dec, plot_height_dec,
                         julia_cx, julia_cy):
    """Parameters of ap_strict_eval as eval_glitched_pixels_fallback_cuda prepares them
    (math_core/engine.py:298-375): x_min, y_max and the pixel steps W-1, H-1 apart in
    Decimal at the view's precision; double-double views of them, or every pixel's c in
    fixed point."""
    from .engine import to_dd
    ctx = decimal_context(plot_width_dec)
    view = abi.ApStrictView()
    view.tier = tier
    q = _copy_params(p)
    q.arith = abi.AP_ARITH_REF_CUDA
    with localcontext(ctx):
        x_min = center_x_dec - (plot_width_dec / Decimal(2))
        y_max = center_y_dec + (plot_height_dec / Decimal(2))
        dx = plot_width_dec / Decimal(max(1, W - 1))
        dy = plot_height_dec / Decimal(max(1, H - 1))
        if tier in (abi.AP_STRICT_DD, abi.AP_STRICT_FP64):
            q.x_min_hi, q.x_min_lo = to_dd(x_min, ctx)
            q.y_max_hi, q.y_max_lo = to_dd(y_max, ctx)
            q.dx_hi, q.dx_lo = to_dd(dx, ctx)
            q.dy_hi, q.dy_lo = to_dd(dy, ctx)
            q.julia_cx_hi, q.julia_cx_lo = to_dd(julia_cx, ctx)
            q.julia_cy_hi, q.julia_cy_lo = to_dd(julia_cy, ctx)
            return q, view, None, None
        n = len(coords)
        signs = np.empty((n, 2), np.int32)
        limbs = np.empty((n, 2, abi.AP_STRICT_NLIMBS), np.uint32)
        for t in range(n):
            signs[t, 0], limbs[t, 0] = fixed_limbs(x_min + Decimal(int(coords[t, 1])) * dx)
            signs[t, 1], limbs[t, 1] = fixed_limbs(y_max - Decimal(int(coords[t, 0])) * dy)
        view.jx_sign, jx = fixed_limbs(Decimal(str(julia_cx)))
        view.jy_sign, jy = fixed_limbs(Decimal(str(julia_cy)))
        view.jx_limbs[:] = [int(x) for x in jx]
        view.jy_limbs[:] = [int(x) for x in jy]
    return q, view, signs, limbs


def strict_values(coords, W, H, max_iter, center_x_dec, center_y_dec, plot_width_dec, plot_height_dec,
                  fractal_type, julia_cx, julia_cy, gen_n, gen_kr, gen_ki, workers=None, scalar=None):
    """Smooth values of the listed (row, col) pixels, each from its own orbit at the
    view's precision: the Strict Metric re-evaluation of math_core/engine.py:191-267
    (its Decimal branch; gmpy2 is not used).  Pixel c is x_min + col dx, y_max - row dy
    in Decimal at int(bits / 3.32) + 30 digits.  ``scalar`` replaces the certified
    native escape evaluation (the exact Decimal one, for instance)."""
    scalar = scalar or hp.compute_highprec_escape_scalar
    from concurrent.futures import ThreadPoolExecutor
    import os
    ctx = decimal_context(plot_width_dec)
    bits = compute_required_prec_bits(plot_width_dec)
    with localcontext(ctx):
        x_min = center_x_dec - (plot_width_dec / Decimal(2))
        y_max = center_y_dec + (plot_height_dec / Decimal(2))
        dx = plot_width_dec * (Decimal(1) / Decimal(max(1, W - 1)))
        dy = plot_height_dec * (Decimal(1) / Decimal(max(1, H - 1)))
    px_ctx = decimal_context()
    px_ctx.prec = int(bits / 3.32) + 30

    def one(rc):
        r, c = int(rc[0]), int(rc[1])
        with localcontext(px_ctx):
            cx = x_min + Decimal(c) * dx
            cy = y_max - Decimal(r) * dy
        return scalar(cx, cy, max_iter, fractal_type, julia_cx, julia_cy, bits,
                      gen_n=gen_n, gen_kr=gen_kr, gen_ki=gen_ki)

    n = workers or min(32, os.cpu_count() or 4)
    with ThreadPoolExecutor(max_workers=n) as ex:
        return np.fromiter(ex.map(one, list(coords)), dtype=np.float64, count=len(coords))


def _copy_params(p):
    q = abi.ApFrameParams()
    C.pointer(q)[0] = p
    return q


def _resolve_params(p, flags, cpu_sem):
    q = _copy_params(p)
    q.flags = flags
    if not cpu_sem:
        q.bla_levels = 0  # the CUDA resolve kernels use the non-BLA sample
    return q
