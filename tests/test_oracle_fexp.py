"""The oracle's FloatExp tier against the reference (tests/golden/fexp_samples.npz).

  * reference orbits at widths below 1e-300 (find_optimal_reference_orbit with
    is_floatexp=True, math_core/high_precision.py:919-1097) match the goldens;
  * per-sample values of cpu_compute_perturbation_sample_floatexp
    (math_core/cpu_kernels.py:606-1021), with and without chained BLA, and the
    glitch flags, are bit-identical for Mandelbrot (config 3's centre at 1e-320
    and 1e-1000), Burning Ship, Julia and Multibrot n = 3.
"""
from decimal import Decimal

import numpy as np
import pytest

import oracle
from fractura_b200 import abi, high_precision
from fractura_b200.config import decimal_context
from helpers import load_golden

G, META = load_golden("fexp_samples.npz")
CASES = [m["name"] for m in META]


def case(name):
    return next(m for m in META if m["name"] == name)


@pytest.mark.parametrize("name", CASES)
def test_floatexp_reference_orbit_matches(name):
    m = case(name)
    with __import__("decimal").localcontext(decimal_context(Decimal(m["width"]))):
        pw = Decimal(m["width"])
        ph = pw * (Decimal(m["H"]) / Decimal(m["W"]))
    high_precision.clear_reference_orbit_cache()
    bcx, bcy, u, v, re, im, rl = high_precision.find_optimal_reference_orbit(
        Decimal(m["cx"]), Decimal(m["cy"]), pw, ph, m["max_iter"], m["W"], m["H"],
        fractal_type=m["fractal_type"], julia_cx=m["julia_cx"], julia_cy=m["julia_cy"],
        gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"], is_floatexp=True)
    assert rl == m["ref_len"] and (u, v) == (m["u"], m["v"])
    assert str(bcx) == m["ref_cx"] and str(bcy) == m["ref_cy"]
    assert np.array_equal(re[:rl + 1], G[name + "__re"]) and np.array_equal(im[:rl + 1], G[name + "__im"])


def floatexp_params(m, variant, arith=abi.AP_ARITH_REF_CPU):
    use_bla = variant == "bla" and m["bla_shape"][0] > 1
    return use_bla, abi.new_params(
        width=m["W"], height=m["H"], max_iter=m["max_iter"], fractal_type=m["fractal_type"],
        tier=abi.AP_TIER_FLOATEXP, arith=arith, gen_n=m["gen_n"], gen_kr=m["gen_kr"],
        gen_ki=m["gen_ki"], julia_cx_hi=m["julia_cx"], julia_cy_hi=m["julia_cy"], dx_hi=m["dx"],
        dy_hi=m["dy"], ref_px=m["ref_px"], ref_py=m["ref_py"], ref_cx=float(Decimal(m["ref_cx"])),
        ref_cy=float(Decimal(m["ref_cy"])), ref_len=m["ref_len"], e_scale=m["e_scale"],
        bla_levels=16 if use_bla else 0, strict_glitch=1 if variant == "bla" else 0,
        flags=abi.AP_FLAG_ESCAPE_GLITCH | abi.AP_FLAG_NAN_GUARD)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("variant", ["plain", "bla"])
def test_floatexp_samples_bit_exact(name, variant):
    m = case(name)
    re, im = G[name + "__re"], G[name + "__im"]
    use_bla, p = floatexp_params(m, variant)
    T = oracle.build_bla(re, im, m["ref_len"], m["fractal_type"], 1e-6, 16, m["gen_n"], m["gen_kr"],
                         m["gen_ki"]) if use_bla else None
    st = m["stride"]
    s, g, _ = oracle.pert_grid(p, re, im, T, np.arange(0, m["W"], st, dtype=np.float64),
                               np.arange(0, m["H"], st, dtype=np.float64))
    ref = G[f"{name}__{variant}_s"]
    assert np.mean(ref >= 0) > 0.5  # the case exercises escapes, not just interior
    assert np.array_equal(s.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(g, G[f"{name}__{variant}_g"])
