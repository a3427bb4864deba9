"""Strict Metric fallback on the device (ap_strict_eval) and through the engine.

* ap_strict_eval equals the oracle on the reference-kernel fixtures (34-limb points,
  double-double and fixed-point frames) value for value, colour for colour.
* Whole Strict Metric frames through render_frame_ssaa equal the oracle's in both
  profiles: the CPU path evaluates the remaining glitched pixels on the host, the CUDA
  path in its device tiers (double-double at 2e-14, fixed point at 1e-160).
"""
import ctypes as C
from decimal import Decimal

import numpy as np
import pytest

import oracle
from fractura_b200 import _lib, abi, engine
from fractura_b200 import high_precision as hp
from helpers import load_golden, oracle_pert_frame, rgb_mismatch
from test_oracle_strict import ML_POINTS, SIM, SIM_FRAMES, ml_point_inputs, sim_frame_inputs

pytestmark = pytest.mark.gpu


def device_strict_eval(fr, q, view, coords, signs, limbs):
    """ap_strict_eval on device copies of an oracle frame's buffers; returns (iter, rgb, glitch)."""
    import torch
    dev = "cuda"

    def d(a):
        return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).to(dev)

    it, rgb, gl = d(fr.iter_map), d(fr.rgb), d(fr.glitch_out)
    lut, cdf = d(fr.lut), d(fr.cdf)
    b = abi.ApFrameBuffers()
    for name, t in (("iter_map", it), ("rgb", rgb), ("glitch_out", gl), ("lut", lut), ("cdf", cdf)):
        setattr(b, name, None if t is None else t.data_ptr())
    d_coords = d(np.asarray(coords, np.int32))
    d_signs = d(signs)
    d_limbs = None if limbs is None else d(np.asarray(limbs, np.uint32).view(np.int32))
    L = _lib.load()
    ptr = (lambda t: None if t is None else C.c_void_p(t.data_ptr()))
    _lib.check(L.ap_strict_eval(C.byref(q), C.byref(b), C.byref(view), ptr(d_coords), ptr(d_signs),
                                ptr(d_limbs), int(len(coords)), None), "ap_strict_eval")
    torch.cuda.synchronize()
    return it.cpu().numpy(), rgb.cpu().numpy(), gl.cpu().numpy()


@pytest.mark.parametrize("ft", [0, 1, 2, 3])
def test_fixed_point_points_device_equals_reference(ft):
    pts = [p for p in ML_POINTS if p["ft"] == ft]
    p, view, coords, signs, limbs = ml_point_inputs(pts)
    fr = oracle.Frame(len(pts), 1, lut=np.zeros(2048 * 3, np.float32))
    it, _, _ = device_strict_eval(fr, p, view, coords, signs, limbs)
    want = np.array([q["s"] for q in pts], np.float32)
    assert np.array_equal(it[0].view(np.uint32), want.view(np.uint32)), (it[0], want)


@pytest.mark.parametrize("name", [m["name"] for m in SIM_FRAMES])
def test_device_tier_frames_device_equals_oracle(name):
    m = next(x for x in SIM_FRAMES if x["name"] == name)
    fr, q, view, coords, signs, limbs = sim_frame_inputs(m)
    it, rgb, gl = device_strict_eval(fr, q, view, coords, signs, limbs)
    oracle.strict_eval(q, fr, view, coords, signs, limbs)
    assert np.array_equal(it.view(np.uint32), fr.iter_map.view(np.uint32))
    assert np.array_equal(it.view(np.uint32), SIM[f"frame_{name}__iter"].view(np.uint32))
    assert rgb_mismatch(rgb, fr.rgb)[0] == 0
    assert not gl.any()


STRICT, STRICT_META = load_golden("render_strict.npz")


def engine_frame(m, arith, glitch_mode=None, width=None, W=None, H=None, max_iter=None):
    W = W or m["W"]
    H = H or m["H"]
    hp.clear_reference_orbit_cache()
    it = np.zeros((H, W), np.float32)
    rgb = engine.render_frame_ssaa(
        W, H, max_iter or m["max_iter"], Decimal(m["cx"]), Decimal(m["cy"]), Decimal(width or m["width"]), None,
        color_scheme_id=m["scheme"], precision_mode="1e-300 (Perturbation)", fractal_type=m["fractal_type"],
        julia_cx=m["julia_cx"], julia_cy=m["julia_cy"], bbsa_tol=1e-6, bbsa_order=m["bbsa_order"],
        glitch_mode=glitch_mode or m["glitch_mode"], gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"],
        h_iter_buf=it, arith=arith)
    return it, rgb


@pytest.mark.parametrize("name", [m["name"] for m in STRICT_META])
@pytest.mark.parametrize("arith", ["ref_cpu", "ref_cuda"])
def test_strict_frame_engine_equals_oracle(name, arith):
    m = next(x for x in STRICT_META if x["name"] == name)
    it, rgb = engine_frame(m, arith)
    from fractura_b200.perturbation import LAST_FRAME_STATS
    # the CPU path stops rebasing at 128 glitched pixels and always leaves some here;
    # the CUDA path may clear them all by rebasing
    assert arith == "ref_cuda" or LAST_FRAME_STATS["strict_pixels"] > 0
    fr, _ = oracle_pert_frame(m, arith=0 if arith == "ref_cpu" else 1)
    assert np.array_equal(it.view(np.uint32), fr.iter_map.view(np.uint32)), \
        int((it.view(np.uint32) != fr.iter_map.view(np.uint32)).sum())
    assert rgb_mismatch(rgb, fr.rgb)[0] == 0
    if arith == "ref_cpu":
        assert np.array_equal(it.view(np.uint32), STRICT[name + "__iter"].view(np.uint32))


def test_strict_frame_fixed_point_tier_through_engine():
    """The CUDA path at 1e-160 (the deep view of the 1920x1080 workload, here 64x36):
    pixels left after rebasing go through the 34-limb device tier."""
    G, META = load_golden("render_pert.npz")
    m = dict(next(x for x in META if x["name"] == "cfg3_bla_pauldelbrot"))
    m.update(W=64, H=36, glitch_mode="Strict Metric", max_iter=20000)
    it, rgb = engine_frame(m, "ref_cuda")
    from fractura_b200.perturbation import LAST_FRAME_STATS
    assert LAST_FRAME_STATS["strict_pixels"] > 0 and LAST_FRAME_STATS["strict_tier"] == abi.AP_STRICT_LIMBS
    fr, _ = oracle_pert_frame(m, arith=1)
    assert np.array_equal(it.view(np.uint32), fr.iter_map.view(np.uint32))
    assert rgb_mismatch(rgb, fr.rgb)[0] == 0


@pytest.mark.parametrize("name", [m["name"] for m in SIM_FRAMES])
def test_public_fallback_equals_reference_kernels(name):
    """engine.eval_glitched_pixels_fallback_cuda (the drop-in for math_core/engine.py:270)
    on the views where the reference's own fallback was run (Numba's CUDA simulator):
    the iteration map, RGB and cleared glitch flags equal the reference's."""
    import torch
    from fractura_b200.palette import synthetic_lut
    m = next(x for x in SIM_FRAMES if x["name"] == name)
    W, H = m["W"], m["H"]
    gl = SIM[f"frame_{name}__glitch_in"]
    pw = Decimal(m["width"])
    ph = pw * (Decimal(H) / Decimal(W))
    d_rgb = torch.zeros((H, W, 3), dtype=torch.uint8, device="cuda")
    d_gl = torch.from_numpy(gl.copy()).cuda()
    d_it = torch.full((H, W), -7.0, dtype=torch.float32, device="cuda")
    d_lut = torch.from_numpy(synthetic_lut()).cuda()
    d_cdf = torch.from_numpy(np.ascontiguousarray(SIM[f"frame_{name}__cdf"])).cuda() if m["scheme"] == 11 else None
    engine.eval_glitched_pixels_fallback_cuda(
        d_rgb, d_gl, d_lut, np.argwhere(gl > 0), W, H, m["max_iter"], Decimal(m["cx"]), Decimal(m["cy"]), pw, ph,
        m["scheme"], m["fractal_type"], m["julia_cx"], m["julia_cy"], gen_n=m["gen_n"], gen_kr=m["gen_kr"],
        gen_ki=m["gen_ki"], d_cdf_lut=d_cdf, num_bins=65536 if m["scheme"] == 11 else 2048, d_iter_map=d_it)
    it = d_it.cpu().numpy()
    sel = gl > 0
    assert np.array_equal(it[sel].view(np.uint32), SIM[f"frame_{name}__iter"][sel].view(np.uint32))
    assert rgb_mismatch(d_rgb.cpu().numpy()[sel][None], SIM[f"frame_{name}__rgb"][sel][None])[0] == 0
    assert np.array_equal(d_gl.cpu().numpy(), SIM[f"frame_{name}__glitch_out"])


@pytest.mark.parametrize("ft", [0, 1, 2, 4])
def test_public_fallback_fp64_tier_equals_oracle(ft):
    """At widths >= 1e-12 the fallback iterates in FP64 (the reference's precision tier 0):
    device == oracle, and the values equal the FP64 samples at c = x_min + col dx."""
    import torch
    from fractura_b200.palette import synthetic_lut
    from fractura_b200.perturbation import strict_device_inputs, strict_device_tier
    W, H, mi = 40, 24, 3000
    cx, cy = {0: ("-0.7436", "0.1318"), 1: ("-1.76", "0.03"), 2: ("0.01", "0.3"), 4: ("-0.2", "0.75")}[ft]
    pw = Decimal("1e-11")
    ph = pw * (Decimal(H) / Decimal(W))
    rng = np.random.default_rng(ft + 5)
    coords = np.argwhere(rng.random((H, W)) < 0.3).astype(np.int32)
    jx, jy = (-0.8, 0.156) if ft == 2 else (0.0, 0.0)
    d_rgb = torch.zeros((H, W, 3), dtype=torch.uint8, device="cuda")
    d_gl = torch.ones((H, W), dtype=torch.uint8, device="cuda")
    d_it = torch.full((H, W), -7.0, dtype=torch.float32, device="cuda")
    lut = synthetic_lut()
    engine.eval_glitched_pixels_fallback_cuda(
        d_rgb, d_gl, torch.from_numpy(lut).cuda(), coords, W, H, mi, Decimal(cx), Decimal(cy), pw, ph, 5, ft,
        jx, jy, gen_n=3, gen_kr=0.1, gen_ki=0.2, d_iter_map=d_it)
    fr = oracle.Frame(W, H, lut=lut)
    fr.iter_map[...] = -7.0
    fr.glitch_out[...] = 1
    p = abi.new_params(width=W, height=H, max_iter=mi, fractal_type=ft, scheme_id=5, gen_n=3, gen_kr=0.1,
                       gen_ki=0.2, arith=abi.AP_ARITH_REF_CUDA)
    tier = strict_device_tier(pw, ft)
    assert tier == abi.AP_STRICT_FP64
    q, view, signs, limbs = strict_device_inputs(p, coords, tier, W, H, Decimal(cx), Decimal(cy), pw, ph, jx, jy)
    oracle.strict_eval(q, fr, view, coords, signs, limbs)
    it = d_it.cpu().numpy()
    assert np.array_equal(it.view(np.uint32), fr.iter_map.view(np.uint32))
    assert rgb_mismatch(d_rgb.cpu().numpy(), fr.rgb)[0] == 0
    assert np.array_equal(d_gl.cpu().numpy(), fr.glitch_out)
    assert not fr.glitch_out[coords[:, 0], coords[:, 1]].any()
    q.tier = abi.AP_TIER_FP64
    xs = q.x_min_hi + coords[:, 1].astype(np.float64) * q.dx_hi
    ys = q.y_max_hi - coords[:, 0].astype(np.float64) * q.dy_hi
    for t in range(len(coords)):
        s32, _, _ = oracle.fp64_grid(q, xs[t:t + 1], ys[t:t + 1])
        assert s32[0, 0] == it[coords[t, 0], coords[t, 1]]
