"""Series-approximation ("BBSA") starts against the reference (tests/golden/bbsa_samples.npz).

  * ap_bbsa_coeffs (host code of the library, no GPU needed) reproduces
    compute_bbsa_coeffs (math_core/high_precision.py:537-578) bit for bit (skip
    and all 16 coefficients), for orders 4 and 8 at two tolerances on the
    Mandelbrot (config 3), Julia and Multibrot orbits;
  * perturbation samples started from the series (oracle, the same evaluation
    the device runs) equal cpu_compute_perturbation_sample's values;
  * whole series-started frames equal render_frame_cpu's.
"""
import ctypes as C
from decimal import Decimal

import numpy as np
import pytest

import oracle
from fractura_b200 import _lib, abi
from helpers import load_golden

B, BMETA = load_golden("bbsa_samples.npz")
P, PMETA = load_golden("pert_samples.npz")


def pert_case(name):
    return next(m for m in PMETA if m["name"] == name)


def coeffs(m, order, tol):
    re, im = P[m["name"] + "__re"], P[m["name"] + "__im"]
    out = np.zeros(17, np.float64)
    L = _lib.load()
    _lib.check(L.ap_bbsa_coeffs(re.ctypes.data_as(C.c_void_p), im.ctypes.data_as(C.c_void_p),
                                m["ref_len"], float(Decimal(m["width"])) * 0.75, m["fractal_type"], tol,
                                order, m["gen_n"], m["gen_kr"], m["gen_ki"], 0,
                                out.ctypes.data_as(C.c_void_p)), "ap_bbsa_coeffs")
    return out


@pytest.mark.parametrize("tag", [m["tag"] for m in BMETA])
def test_bbsa_coefficients_match_reference(tag):
    bm = next(x for x in BMETA if x["tag"] == tag)
    m = pert_case(bm["name"])
    got = coeffs(m, bm["order"], bm["tol"])
    ref = B[tag + "__coeffs"]
    assert int(got[0]) == int(ref[0]) == bm["skip"]
    # bit for bit: the library evaluates the recurrence in the rounding order of the
    # reference's compiled fast-math kernel
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64)), \
        np.max(np.abs(got[1:] - ref[1:]) / np.maximum(np.abs(ref[1:]), 1e-300))


def test_bbsa_disabled_cases_return_zero():
    m = pert_case("ship")  # Burning Ship: no series start
    assert not np.any(coeffs(m, 4, 1e-4))
    m = pert_case("cfg3")
    assert not np.any(coeffs(m, 32, 1e-6))  # chained BLA selects no series start


@pytest.mark.parametrize("tag", [m["tag"] for m in BMETA if m["tol"] == 1e-4])
def test_series_started_samples_bit_exact(tag):
    bm = next(x for x in BMETA if x["tag"] == tag)
    m = pert_case(bm["name"])
    ref_s = B[tag + "__s"]
    st = int(B[tag + "__stride"][0])
    c = B[tag + "__coeffs"]
    p = abi.new_params(width=m["W"], height=m["H"], max_iter=m["max_iter"], fractal_type=m["fractal_type"],
                       tier=abi.AP_TIER_PERTURB, arith=abi.AP_ARITH_REF_CPU, gen_n=m["gen_n"],
                       gen_kr=m["gen_kr"], gen_ki=m["gen_ki"], julia_cx_hi=m["julia_cx"],
                       julia_cy_hi=m["julia_cy"], dx_hi=m["dx"], dy_hi=m["dy"], ref_px=m["ref_px"],
                       ref_py=m["ref_py"], ref_cx=float(Decimal(m["ref_cx"])),
                       ref_cy=float(Decimal(m["ref_cy"])), ref_len=m["ref_len"], bla_levels=0,
                       strict_glitch=0, bbsa_skip=int(c[0]), bbsa_inv_r=1.0 / bm["max_r"],
                       bbsa=list(c[1:17]), flags=abi.AP_FLAG_ESCAPE_GLITCH | abi.AP_FLAG_NAN_GUARD)
    s, _, _ = oracle.pert_grid(p, P[m["name"] + "__re"], P[m["name"] + "__im"], None,
                               np.arange(0, m["W"], st, dtype=np.float64),
                               np.arange(0, m["H"], st, dtype=np.float64))
    assert np.array_equal(s.view(np.uint32), ref_s.view(np.uint32)), \
        int((s.view(np.uint32) != ref_s.view(np.uint32)).sum())


# Whole frames (rebasing included) with the engine's own coefficients equal
# render_frame_cpu's value for value, the ill-conditioned Multibrot n = 3 view too.
R, RMETA = load_golden("render_bbsa.npz")


@pytest.mark.parametrize("name", [m["name"] for m in RMETA])
def test_series_started_frames_against_reference(name):
    from helpers import oracle_pert_frame
    m = next(x for x in RMETA if x["name"] == name)
    fr, _ = oracle_pert_frame(m)
    ref = R[name + "__iter"]
    assert np.array_equal(fr.iter_map.view(np.uint32), ref.view(np.uint32)), \
        int((fr.iter_map.view(np.uint32) != ref.view(np.uint32)).sum())


@pytest.mark.parametrize("tag", [m["tag"] for m in BMETA])
def test_engine_compute_bbsa_coeffs_cuda_matches_reference(tag):
    """engine.compute_bbsa_coeffs_cuda (the drop-in for math_core/engine.py:426) returns
    the reference's (skip, 16 coefficients) tuple, bit for bit, from device or host arrays."""
    from fractura_b200 import engine
    bm = next(x for x in BMETA if x["tag"] == tag)
    m = pert_case(bm["name"])
    re, im = P[m["name"] + "__re"], P[m["name"] + "__im"]
    got = engine.compute_bbsa_coeffs_cuda(re, im, m["ref_len"], float(Decimal(m["width"])) * 0.75,
                                          m["fractal_type"], bbsa_tol=bm["tol"], bbsa_order=bm["order"],
                                          gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"],
                                          h_ref_re=re, h_ref_im=im)
    ref = B[tag + "__coeffs"]
    assert got[0] == int(ref[0]) and isinstance(got[0], int)
    assert np.array_equal(np.array(got[1:], np.float64).view(np.uint64), ref[1:].view(np.uint64))


def test_engine_compute_bbsa_coeffs_cuda_guards():
    from fractura_b200 import engine
    m = pert_case("cfg3")
    re, im = P["cfg3__re"], P["cfg3__im"]
    zero = (0,) + (0.0,) * 16
    assert engine.compute_bbsa_coeffs_cuda(re, im, m["ref_len"], 1e-160, 1) == zero          # Burning Ship
    assert engine.compute_bbsa_coeffs_cuda(re, im, m["ref_len"], 1e-160, 0, bbsa_order=32) == zero
    assert engine.compute_bbsa_coeffs_cuda(re, im, 1, 1e-160, 0) == zero                     # ref_len < 2
    assert engine.compute_bbsa_coeffs_cuda(re, im, m["ref_len"], 0.0, 0) == zero             # max_r <= 0
