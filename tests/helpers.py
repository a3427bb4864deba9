"""Shared helpers of the test-suite: golden fixtures and oracle frames."""
import json
import math
import os
from decimal import Decimal, localcontext

import numpy as np

import oracle
import ref_orbit
from fractura_b200 import abi
from fractura_b200.config import compute_floatexp_scale, decimal_context
from fractura_b200.engine import plan_direct_view
from fractura_b200.palette import synthetic_lut

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    g = np.load(os.path.join(GOLDEN, name))
    return g, json.loads(str(g["meta"]))


def direct_params(m, tier=abi.AP_TIER_FP64, arith=abi.AP_ARITH_REF_CPU):
    """ApFrameParams of a render case dict (keys as in make_golden.RENDER1_CASES)."""
    W, H, f = m["W"], m["H"], m["factor"]
    view = plan_direct_view(W, H, f, Decimal(m["cx"]), Decimal(m["cy"]), Decimal(m["width"]), tier,
                            m.get("julia_cx", 0.0), m.get("julia_cy", 0.0))
    p = abi.new_params(width=W, height=H, factor=f, max_iter=m["max_iter"],
                       fractal_type=m["fractal_type"], tier=tier, arith=arith,
                       gen_n=m.get("gen_n", 3), gen_kr=m.get("gen_kr", 0.25), gen_ki=m.get("gen_ki", 1.0),
                       scheme_id=m["scheme"], palette_offset=m.get("offset", 0.0),
                       color_density=m.get("density", 1.0), color_contrast=m.get("contrast", 1.0),
                       num_bins=65536 if m["scheme"] == 11 else 2048)
    for k, v in view.items():
        setattr(p, k, v)
    return p


def oracle_direct_frame(m, tier=abi.AP_TIER_FP64, arith=abi.AP_ARITH_REF_CPU, lut=None,
                        edge_threshold=0.35):
    """Full frame through the oracle, in the order the engine issues its passes."""
    p = direct_params(m, tier, arith)
    fr = oracle.Frame(m["W"], m["H"], lut=synthetic_lut() if lut is None else lut)
    cpu = arith == abi.AP_ARITH_REF_CPU
    f = m["factor"]
    if m["scheme"] == 11:
        p.flags = abi.AP_FLAG_NO_RGB
        oracle.render_pass(p, fr)
        oracle.histogram_cdf(fr, m["max_iter"])
        oracle.colour(p, fr)
        if f > 1:
            oracle.edge_detect(fr, np.float32(edge_threshold))
            p.flags = abi.AP_FLAG_MAP_FUSED if cpu else 0
            oracle.resolve_hist_pass(p, fr)
    else:
        p.flags = abi.AP_FLAG_MAP_FUSED if cpu else 0
        oracle.render_pass(p, fr)
        if f > 1:
            oracle.edge_detect(fr, np.float32(edge_threshold))
            p.mode = abi.AP_MODE_EDGE
            oracle.render_pass(p, fr)
    return fr


def rgb_mismatch(a, b):
    diff = np.abs(a.astype(np.int64) - b.astype(np.int64))
    return int(diff.any(axis=-1).sum()), int(diff.max()) if diff.size else 0


def oracle_pert_frame(m, arith=abi.AP_ARITH_REF_CPU, lut=None, edge_threshold=0.35, max_passes=4,
                      bla_eps=None):
    """A perturbation-tier frame through the oracle, pass for pass as the engine issues it
    (fractura_b200.perturbation.render_perturbation_frame), including the rebase loop.
    ``bla_eps`` selects the dc-aware BLA table (the engine's bla_form="accurate")."""
    from fractura_b200.config import compute_required_prec_bits
    from fractura_b200.perturbation import RebaseState, max_delta_c, select_rebase_pixel
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
    # the oracle's own Decimal restatement of the reference's orbit search (oracle/ref_orbit.py)
    bcx, bcy, bu, bv, re, im, rl = ref_orbit.find_reference(
        cxd, cyd, pw, ph, mi, ft=ft, julia_cx=m["julia_cx"], julia_cy=m["julia_cy"],
        n=m["gen_n"], kr=m["gen_kr"], ki=m["gen_ki"])
    order = m["bbsa_order"]
    if floatexp and order in (4, 8):
        order = 32  # the reference maps series starts to chained BLA on this tier
    # Series-start coefficients come from the library's host function, which
    # tests/test_bbsa.py pins against the reference's compute_bbsa_coeffs.
    from fractura_b200 import _lib
    from fractura_b200.perturbation import bbsa_coefficients
    max_r = float(pw) * 0.75
    inv_r = 1.0 / max_r if max_r > 0.0 else 1.0
    bbsa_tol = m.get("bbsa_tol", 1e-4)

    def series(r_re, r_im, r_len):
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
    one_pass = "One-Pass Rebasing" in m["glitch_mode"]
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
        oracle.render_pass(p, fr)
        oracle.histogram_cdf(fr, mi)
        oracle.colour(p, fr)
        if f > 1:
            oracle.edge_detect(fr, np.float32(edge_threshold))
            q = abi.ApFrameParams.from_buffer_copy(p)
            resolve(q)
    else:
        p.flags = uf
        oracle.render_pass(p, fr)
        if f > 1:
            oracle.edge_detect(fr, np.float32(edge_threshold))
            p.mode = abi.AP_MODE_EDGE
            p.flags = uf | (0 if cpu_sem else abi.AP_FLAG_ITER_LAST_SUB)
            oracle.render_pass(p, fr)
    if not (strict and pw < Decimal("1e-12")):
        return fr, 0
    state = RebaseState((int(np.clip(p.ref_py / f, 0, H - 1)), int(np.clip(p.ref_px / f, 0, W - 1))),
                        "Strict" in m["glitch_mode"], 128 if cpu_sem else 512)
    bits = compute_required_prec_bits(pw)
    while state.passes < max_passes:
        g = fr.glitch_out.copy()
        if not state.should_continue(int(np.count_nonzero(g))):
            break
        state.passes += 1
        chosen = select_rebase_pixel(g, fr.iter_map, mi, state.visited, W, H)
        if chosen is None:
            break
        state.visited.add(chosen)
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
            oracle.render_pass(q, fr)
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
                                 m["gen_n"], m["gen_kr"], m["gen_ki"], scalar=_oracle_escape)
            q = abi.ApFrameParams.from_buffer_copy(p)
            q.arith = abi.AP_ARITH_REF_CPU
            oracle.set_pixels(q, fr, coords, vals)
        elif len(coords):
            q, view, signs, limbs = strict_device_inputs(p, coords, tier, W, H, cxd, cyd, pw, ph, m["julia_cx"],
                                                         m["julia_cy"])
            oracle.strict_eval(q, fr, view, coords, signs, limbs)
    return fr, state.passes


def _oracle_escape(cx, cy, max_iter, fractal_type, julia_cx, julia_cy, bits, gen_n=3, gen_kr=0.25, gen_ki=1.0):
    """The Strict Metric's host value of one pixel through the oracle's Decimal restatement."""
    return ref_orbit.escape(cx, cy, max_iter, fractal_type, julia_cx, julia_cy, bits, n=gen_n, kr=gen_kr,
                            ki=gen_ki)


def probe_search(base_iter):
    """Probe depth searched for a base depth (math_core/engine.py:1069)."""
    from fractura_b200.config import GLOBAL_MAX_ITER
    return min(GLOBAL_MAX_ITER, max(1000, int(base_iter * 2)))


def probe_args(m):
    """Positional arguments of engine.plan_probe / probe_iter_map for a probe case."""
    return (Decimal(m["cx"]), Decimal(m["cy"]), Decimal(m["width"]), probe_search(m["base_iter"]),
            m["W"], m["H"], m["fractal_type"], m["julia_cx"], m["julia_cy"], m["gen_n"], m["gen_kr"],
            m["gen_ki"], m["precision_mode"], m["bbsa_tol"], m["bbsa_order"])


def oracle_probe(m, arith=abi.AP_ARITH_REF_CPU):
    """Probe map of a probe case through the oracle, on the pass engine.plan_probe plans."""
    from fractura_b200 import engine
    from fractura_b200 import high_precision as hp
    hp.clear_reference_orbit_cache()
    p, orbit = engine.plan_probe(*probe_args(m), arith=arith)
    fr = oracle.Frame(m["W"], m["H"], lut=synthetic_lut())
    if orbit is not None:
        re, im, rl = orbit
        fr.ref_re, fr.ref_im = np.ascontiguousarray(re[:rl + 1]), np.ascontiguousarray(im[:rl + 1])
    oracle.render_pass(p, fr)
    return fr.iter_map
