"""The oracle's FP32-mantissa FloatExp form (AP_TIER_FLOATEXP32) against the reference.

The form is the engine's own (24-bit delta mantissas with int exponents, FP64 tests); the
oracle restates it from its definition so that device frames can be compared with it bit
for bit (tests/test_gpu_fe32.py).  Where 24 bits carry the view -- the reference's
FloatExp goldens (tests/golden/fexp_samples.npz: Mandelbrot at 1e-320 and 1e-1000,
Burning Ship and Multibrot n = 3 at 1e-320, Julia at 1e-400) -- the form's samples equal
the reference's own cpu_compute_perturbation_sample_floatexp values
(math_core/cpu_kernels.py:606-1021) bit for bit: the float32 smooth value, the escape
step and the Pauldelbrot flag, with and without chained-BLA leaps, and with one-pass
rebasing in place of the flags.
"""
import numpy as np
import pytest

import oracle
from fractura_b200 import abi
from test_oracle_fexp import G, META, floatexp_params

CASES = [m["name"] for m in META]


def fe32_grid(m, variant, one_pass=False):
    re, im = G[m["name"] + "__re"], G[m["name"] + "__im"]
    use_bla, p = floatexp_params(m, variant, arith=abi.AP_ARITH_REF_CUDA)
    p.tier = abi.AP_TIER_FLOATEXP32
    p.flags = abi.AP_FLAG_NAN_GUARD | (abi.AP_FLAG_REBASE if one_pass else 0)
    if one_pass:
        p.strict_glitch = 0
    T = oracle.build_bla(re, im, m["ref_len"], m["fractal_type"], 1e-6, 16, m["gen_n"], m["gen_kr"],
                         m["gen_ki"]) if use_bla else None
    st = m["stride"]
    return oracle.pert_grid(p, re, im, T, np.arange(0, m["W"], st, dtype=np.float64),
                            np.arange(0, m["H"], st, dtype=np.float64))


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("variant", ["plain", "bla"])
def test_fe32_samples_equal_the_reference_floatexp_samples(name, variant):
    m = next(x for x in META if x["name"] == name)
    s, g, k = fe32_grid(m, variant)
    ref = G[f"{name}__{variant}_s"]
    assert np.mean(ref >= 0) > 0.5
    assert np.array_equal(s.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(g, G[f"{name}__{variant}_g"])


@pytest.mark.parametrize("name", [m["name"] for m in META if m["fractal_type"] in (0, 1, 4)])
@pytest.mark.parametrize("variant", ["plain", "bla"])
def test_fe32_one_pass_samples_equal_the_reference_samples(name, variant):
    """One-pass rebasing: no sample is flagged, and every value is the reference's."""
    m = next(x for x in META if x["name"] == name)
    s, g, k = fe32_grid(m, variant, one_pass=True)
    assert not g.any()
    assert np.array_equal(s.view(np.uint32), G[f"{name}__{variant}_s"].view(np.uint32))


def test_fe32_renormalisation_keeps_the_escape_step():
    """The same samples with the pixel offsets expressed at another power-of-two scale
    (E + 40, spacing times 2^40): the float mantissas are the same, only the exponents
    move, so every escape step and smooth value is unchanged."""
    m = next(x for x in META if x["name"] == "fexp_mandel")
    s0, _, _ = fe32_grid(m, "plain")
    re, im = G["fexp_mandel__re"], G["fexp_mandel__im"]
    _, p = floatexp_params(m, "plain", arith=abi.AP_ARITH_REF_CUDA)
    p.tier = abi.AP_TIER_FLOATEXP32
    p.flags = abi.AP_FLAG_NAN_GUARD
    p.e_scale += 40
    p.dx_hi *= 2.0 ** 40
    p.dy_hi *= 2.0 ** 40
    st = m["stride"]
    s1, _, _ = oracle.pert_grid(p, re, im, None, np.arange(0, m["W"], st, dtype=np.float64),
                                np.arange(0, m["H"], st, dtype=np.float64))
    assert np.array_equal(s0.view(np.uint32), s1.view(np.uint32))
