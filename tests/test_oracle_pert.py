"""Perturbation inputs and samples against the reference (CPU only).

  * host reference orbits (fractura_b200.high_precision) reproduce the
    reference's Decimal orbits, escape step and 16-candidate choice exactly;
  * the oracle's chained-BLA table is byte-identical to _jit_build_bla_table;
  * the oracle's FP64-delta perturbation samples equal
    cpu_compute_perturbation_sample's, with and without BLA leaps.
"""
import ctypes as C
import hashlib
from decimal import Decimal

import numpy as np
import pytest

import oracle
from fractura_b200 import abi, high_precision
from fractura_b200.config import decimal_context
from helpers import load_golden

G, META = load_golden("pert_samples.npz")
CASES = [m["name"] for m in META]


def case(name):
    return next(m for m in META if m["name"] == name)


def orbit_of(m):
    with __import__("decimal").localcontext(decimal_context(Decimal(m["width"]))):
        pw = Decimal(m["width"])
        ph = pw * (Decimal(m["H"]) / Decimal(m["W"]))
    high_precision.clear_reference_orbit_cache()
    return high_precision.find_optimal_reference_orbit(
        Decimal(m["cx"]), Decimal(m["cy"]), pw, ph, m["max_iter"], m["W"], m["H"],
        fractal_type=m["fractal_type"], julia_cx=m["julia_cx"], julia_cy=m["julia_cy"],
        gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"])


@pytest.mark.parametrize("name", CASES)
def test_reference_orbit_matches(name):
    m = case(name)
    bcx, bcy, u, v, re, im, rl = orbit_of(m)
    assert rl == m["ref_len"] and (u, v) == (m["u"], m["v"])
    assert str(bcx) == m["ref_cx"] and str(bcy) == m["ref_cy"]
    assert np.array_equal(re[:rl + 1], G[name + "__re"]) and np.array_equal(im[:rl + 1], G[name + "__im"])


def bla_table(m, re, im):
    levels, L = m["bla_shape"][0], m["bla_shape"][1]
    T = np.zeros((levels, L, 5), np.float64)
    rc = oracle.lib().apo_build_bla(oracle.ptr(np.ascontiguousarray(re)), oracle.ptr(np.ascontiguousarray(im)),
                                    m["ref_len"], m["fractal_type"], C.c_double(1e-6), levels, m["gen_n"],
                                    C.c_double(m["gen_kr"]), C.c_double(m["gen_ki"]), oracle.ptr(T))
    assert rc == 0
    return T


@pytest.mark.parametrize("name", CASES)
def test_bla_table_byte_identical(name):
    m = case(name)
    if m["bla_shape"][0] <= 1:
        pytest.skip("no BLA table for this formula")
    T = bla_table(m, G[name + "__re"], G[name + "__im"])
    assert hashlib.sha256(T.tobytes()).digest() == G[name + "__bla_sha256"].tobytes()


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("variant", ["plain", "bla"])
def test_perturbation_samples_bit_exact(name, variant):
    m = case(name)
    re, im = G[name + "__re"], G[name + "__im"]
    use_bla = variant == "bla" and m["bla_shape"][0] > 1
    T = bla_table(m, re, im) if use_bla else None
    H, W, st = m["H"], m["W"], m["stride"]
    p = abi.new_params(width=W, height=H, max_iter=m["max_iter"], fractal_type=m["fractal_type"],
                       tier=abi.AP_TIER_PERTURB, arith=abi.AP_ARITH_REF_CPU, gen_n=m["gen_n"],
                       gen_kr=m["gen_kr"], gen_ki=m["gen_ki"], julia_cx_hi=m["julia_cx"],
                       julia_cy_hi=m["julia_cy"], dx_hi=m["dx"], dy_hi=m["dy"], ref_px=m["ref_px"],
                       ref_py=m["ref_py"], ref_cx=float(Decimal(m["ref_cx"])),
                       ref_cy=float(Decimal(m["ref_cy"])), ref_len=m["ref_len"],
                       bla_levels=m["bla_shape"][0] if use_bla else 0,
                       strict_glitch=1 if variant == "bla" else 0,
                       flags=abi.AP_FLAG_ESCAPE_GLITCH | abi.AP_FLAG_NAN_GUARD)
    s, g, _ = oracle.pert_grid(p, re, im, T, np.arange(0, W, st, dtype=np.float64),
                            np.arange(0, H, st, dtype=np.float64))
    assert np.array_equal(s.view(np.uint32), G[f"{name}__{variant}_s"].view(np.uint32))
    assert np.array_equal(g, G[f"{name}__{variant}_g"])
