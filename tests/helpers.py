"""Shared helpers of the test-suite: golden fixtures and oracle frames."""
import json
import math
import os
from decimal import Decimal, localcontext

import numpy as np

import frames
import oracle
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
                      bla_eps=None, fp32=False):
    """A perturbation-tier frame through the oracle (oracle/frames.py), including the
    rebase loop: (frame, rebase passes).  ``fp32``: the FP32-mantissa form on coarse passes."""
    return frames.pert_frame(m, arith=arith, lut=lut, edge_threshold=edge_threshold, max_passes=max_passes,
                             bla_eps=bla_eps, fp32=fp32)


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
