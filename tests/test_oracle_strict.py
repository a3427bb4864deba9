"""Strict Metric frames through the oracle against render_frame_cpu -- CPU only.

After the rebase loop (which stops at 128 glitched pixels on the CPU path), every pixel
still flagged is evaluated on its own orbit at the view's precision and written back with
its colour (math_core/engine.py:191-267, :1033-1046).  The oracle does the same with the
exact Decimal escape evaluation, so iteration maps must be bit-identical.

The CUDA path evaluates those pixels on the device instead, in double-double or in
34-limb fixed point; those tiers are pinned to the reference's kernels run in Numba's
CUDA simulator (tests/golden/make_golden_cudasim.py)."""
import json
import os
from decimal import Decimal

import numpy as np
import pytest

import oracle
from helpers import GOLDEN, load_golden, oracle_pert_frame, rgb_mismatch
from fractura_b200 import abi

G, META = load_golden("render_strict.npz")


@pytest.mark.parametrize("name", [m["name"] for m in META])
def test_strict_frame_matches_reference(name):
    m = next(x for x in META if x["name"] == name)
    fr, _ = oracle_pert_frame(m)
    ref_it = G[name + "__iter"]
    diff = fr.iter_map.view(np.uint32) != ref_it.view(np.uint32)
    assert not diff.any(), int(diff.sum())
    n_bad, max_diff = rgb_mismatch(fr.rgb, G[name + "__rgb"])
    assert n_bad == 0, (n_bad, max_diff)
    assert not fr.glitch_out.any()


def test_strict_frames_exercise_the_fallback():
    """Each fixture leaves glitched pixels after rebasing, so the fallback is what is tested:
    the same frame without the Strict step differs from the reference."""
    m = dict(next(x for x in META if x["name"] == "strict_ship"))
    m["glitch_mode"] = "Pauldelbrot"
    fr, _ = oracle_pert_frame(m)
    assert fr.glitch_out.any()
    assert (fr.iter_map.view(np.uint32) != G["strict_ship__iter"].view(np.uint32)).any()


def test_set_pixels_writes_value_colour_and_clears_flag():
    W, H = 5, 3
    lut = np.linspace(0, 255, 2048 * 3, dtype=np.float32)
    fr = oracle.Frame(W, H, lut=lut)
    fr.glitch_out[...] = 1
    p = abi.new_params(width=W, height=H, max_iter=100, scheme_id=0)
    coords = np.array([[0, 0], [2, 4], [1, 2], [5, 0]], np.int32)  # the last is outside: skipped
    vals = np.array([12.5, 100.0, -1.0, 3.0])
    oracle.set_pixels(p, fr, coords, vals)
    assert fr.iter_map[0, 0] == np.float32(12.5) and fr.iter_map[2, 4] == 100.0 and fr.iter_map[1, 2] == -1.0
    assert fr.rgb[0, 0].any() and not fr.rgb[2, 4].any() and not fr.rgb[1, 2].any()
    assert fr.glitch_out.sum() == W * H - 3


# ---------------------------------------------------------------------------
# Device tiers of the CUDA path's fallback (double-double, 34-limb fixed point)
# ---------------------------------------------------------------------------
SIM = np.load(os.path.join(GOLDEN, "strict_cuda.npz"))
ML_POINTS = json.loads(str(SIM["ml"]))
SIM_FRAMES = json.loads(str(SIM["frames"]))


def test_fixed_limbs_match_reference_conversion():
    from fractura_b200.perturbation import fixed_limbs
    for pt in ML_POINTS:
        for key, sk, lk in (("x", "sx", "lx"), ("y", "sy", "ly")):
            s, limbs = fixed_limbs(Decimal(pt[key]))
            assert s == pt[sk] and limbs.tolist() == pt[lk], (pt[key], key)


def ml_point_inputs(points):
    """One row of pixels, pixel t = point t, with its limbs and the Julia constant."""
    from fractura_b200.perturbation import fixed_limbs
    n = len(points)
    signs = np.array([[p["sx"], p["sy"]] for p in points], np.int32)
    limbs = np.array([[p["lx"], p["ly"]] for p in points], np.uint32)
    view = abi.ApStrictView()
    view.tier = abi.AP_STRICT_LIMBS
    p0 = points[0]
    if p0["ft"] in (2, 3):
        view.jx_sign, jx = fixed_limbs(Decimal(str(p0["jx"])))
        view.jy_sign, jy = fixed_limbs(Decimal(str(p0["jy"])))
        view.jx_limbs[:] = [int(v) for v in jx]
        view.jy_limbs[:] = [int(v) for v in jy]
    coords = np.stack([np.zeros(n, np.int32), np.arange(n, dtype=np.int32)], axis=1)
    p = abi.new_params(width=n, height=1, max_iter=p0["max_iter"], fractal_type=p0["ft"], scheme_id=0,
                       arith=abi.AP_ARITH_REF_CUDA)
    return p, view, coords, signs, limbs


@pytest.mark.parametrize("ft", [0, 1, 2, 3])
def test_fixed_point_tier_matches_reference_kernel(ft):
    pts = [p for p in ML_POINTS if p["ft"] == ft]
    p, view, coords, signs, limbs = ml_point_inputs(pts)
    fr = oracle.Frame(len(pts), 1, lut=np.zeros(2048 * 3, np.float32))
    oracle.strict_eval(p, fr, view, coords, signs, limbs)
    want = np.array([q["s"] for q in pts], np.float32)
    assert np.array_equal(fr.iter_map[0].view(np.uint32), want.view(np.uint32)), (fr.iter_map[0], want)


def sim_frame_inputs(m):
    from fractura_b200.perturbation import strict_device_inputs, strict_device_tier
    from fractura_b200.palette import synthetic_lut
    W, H = m["W"], m["H"]
    gl = SIM[f"frame_{m['name']}__glitch_in"]
    fr = oracle.Frame(W, H, lut=synthetic_lut())
    fr.iter_map[...] = -7.0
    fr.glitch_out[...] = gl
    if m["scheme"] == 11:
        fr.cdf = np.ascontiguousarray(SIM[f"frame_{m['name']}__cdf"])
    p = abi.new_params(width=W, height=H, max_iter=m["max_iter"], fractal_type=m["fractal_type"],
                       scheme_id=m["scheme"], num_bins=65536 if m["scheme"] == 11 else 2048,
                       gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"], arith=abi.AP_ARITH_REF_CUDA,
                       palette_offset=0.0, color_density=1.0, color_contrast=1.0)
    pw = Decimal(m["width"])
    ph = pw * (Decimal(H) / Decimal(W))
    coords = np.argwhere(gl > 0)
    tier = strict_device_tier(pw, m["fractal_type"])
    q, view, signs, limbs = strict_device_inputs(p, coords, tier, W, H, Decimal(m["cx"]), Decimal(m["cy"]), pw, ph,
                                                 m["julia_cx"], m["julia_cy"])
    return fr, q, view, coords, signs, limbs


@pytest.mark.parametrize("name", [m["name"] for m in SIM_FRAMES])
def test_device_tier_frame_matches_reference(name):
    m = next(x for x in SIM_FRAMES if x["name"] == name)
    fr, q, view, coords, signs, limbs = sim_frame_inputs(m)
    assert view.tier == (abi.AP_STRICT_DD if name.startswith("dd_") else abi.AP_STRICT_LIMBS)
    oracle.strict_eval(q, fr, view, coords, signs, limbs)
    want = SIM[f"frame_{name}__iter"]
    assert np.array_equal(fr.iter_map.view(np.uint32), want.view(np.uint32)), \
        int((fr.iter_map.view(np.uint32) != want.view(np.uint32)).sum())
    n_bad, max_diff = rgb_mismatch(fr.rgb, SIM[f"frame_{name}__rgb"])
    assert n_bad == 0, (n_bad, max_diff)
    assert np.array_equal(fr.glitch_out, SIM[f"frame_{name}__glitch_out"])
