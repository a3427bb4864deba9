"""One-pass rebasing on the device (AP_FLAG_REBASE): the engine's glitch mode
"One-Pass Rebasing".

* Config 3 at full size (1920x1080, width 1e-160, max_iter 200000, FP64 deltas with the
  dc-aware chained BLA): smooth error p99 <= 1e-4 and an identical escape step on
  >= 99.9 % of the 700-bit ground truth's 64 x 64 samples, no pixel glitched, no
  re-render pass, and the device's values equal the oracle's bit for bit there.
* Frames of every served formula, both arithmetic profiles, with and without BLA, at
  factor 1 (packed coarse kernel), with 2x SSAA (generic edge pass) and with histogram
  colouring: iteration map and RGB equal the oracle's frame.
"""
import ctypes as C
from decimal import Decimal

import numpy as np
import pytest

import oracle
from fractura_b200 import _lib, abi, engine, perturbation
from fractura_b200 import high_precision as hp
from fractura_b200.perturbation import ONE_PASS_REBASING, max_delta_c
from helpers import GOLDEN, load_golden, oracle_pert_frame, rgb_mismatch

pytestmark = pytest.mark.gpu

PS, PMETA = load_golden("pert_samples.npz")
RS, RMETA = load_golden("render_pert.npz")

P99_BOUND = 1e-4
K_IDENTICAL_BOUND = 0.999
ARITH = {"ref_cpu": abi.AP_ARITH_REF_CPU, "ref_cuda": abi.AP_ARITH_REF_CUDA, "fast": abi.AP_ARITH_FAST}


@pytest.mark.parametrize("arith", ["ref_cpu", "ref_cuda", "fast"])
def test_config3_one_pass_frame_meets_accuracy_bound(arith):
    import torch
    m = next(x for x in PMETA if x["name"] == "cfg3")
    W, H = m["W"], m["H"]
    t = np.load(f"{GOLDEN}/truth_cfg3.npz")
    truth, rows, cols = t["s"], t["rows"], t["cols"]
    kmap = torch.empty((H, W), dtype=torch.int32, device="cuda")
    s64 = torch.empty((H, W), dtype=torch.float64, device="cuda")
    hp.clear_reference_orbit_cache()
    engine.render_frame_ssaa(W, H, m["max_iter"], Decimal(m["cx"]), Decimal(m["cy"]), Decimal(m["width"]),
                             None, precision_mode="1e-300 (Perturbation)", bbsa_order=32, bbsa_tol=1e-6,
                             glitch_mode=ONE_PASS_REBASING, bla_form="accurate", arith=arith,
                             _extra_out=(kmap, s64))
    assert perturbation.LAST_FRAME_STATS["rebase_passes"] == 0
    k = kmap.cpu().numpy()[np.ix_(rows, cols)]
    s = s64.cpu().numpy()[np.ix_(rows, cols)]
    err = np.abs(s - truth)
    p99, kid = float(np.percentile(err, 99)), float(np.mean(k == np.floor(truth)))
    assert p99 <= P99_BOUND, (p99, kid, float(err.max()))
    assert kid >= K_IDENTICAL_BOUND, (p99, kid, float(err.max()))
    # the same samples through the oracle, on the reference's own orbit and view
    re, im, rl = PS["cfg3__re"], PS["cfg3__im"], m["ref_len"]
    dcm = max_delta_c(m["ref_px"], m["ref_py"], W, H, m["dx"], m["dy"])
    T = oracle.build_bla_dc(re, im, rl, 0, engine.ACCURATE_BLA_EPS, dcm, 16, 3, 0.25, 1.0)
    p = abi.new_params(width=W, height=H, max_iter=m["max_iter"], tier=abi.AP_TIER_PERTURB,
                       arith=ARITH[arith],
                       dx_hi=m["dx"], dy_hi=m["dy"], ref_px=m["ref_px"], ref_py=m["ref_py"], ref_len=rl,
                       bla_levels=16, flags=abi.AP_FLAG_REBASE)
    _, g, ko, so = oracle.pert_grid(p, re, im, T, cols.astype(np.float64), rows.astype(np.float64),
                                    with_s64=True)
    assert not g.any()
    assert np.array_equal(ko, k)
    assert np.array_equal(so.view(np.uint64), s.view(np.uint64))


FRAME_CASES = ["cfg3_bla_pauldelbrot", "cfg3_plain", "cfg3_hist", "cfg3_ssaa2", "cfg3_hist_ssaa2",
               "ship_frame", "multibrot3_frame"]


@pytest.mark.parametrize("name", FRAME_CASES)
@pytest.mark.parametrize("arith", ["ref_cpu", "ref_cuda", "fast"])
@pytest.mark.parametrize("bla_form", ["reference", "accurate"])
def test_one_pass_frames_match_oracle(name, arith, bla_form):
    import torch
    m = dict(next(x for x in RMETA if x["name"] == name))
    m["glitch_mode"] = ONE_PASS_REBASING
    W, H = m["W"], m["H"]
    hp.clear_reference_orbit_cache()
    it = np.zeros((H, W), np.float32)
    kmap = torch.empty((H, W), dtype=torch.int32, device="cuda")
    s64 = torch.empty((H, W), dtype=torch.float64, device="cuda")
    rgb = engine.render_frame_ssaa(
        W, H, m["max_iter"], Decimal(m["cx"]), Decimal(m["cy"]), Decimal(m["width"]), None,
        ssaa_factor=m["factor"], color_scheme_id=m["scheme"], precision_mode="1e-300 (Perturbation)",
        fractal_type=m["fractal_type"], bbsa_tol=1e-6 if m["bbsa_order"] == 32 else 0.0,
        bbsa_order=m["bbsa_order"], glitch_mode=ONE_PASS_REBASING, gen_n=m["gen_n"], gen_kr=m["gen_kr"],
        gen_ki=m["gen_ki"], h_iter_buf=it, arith=arith, bla_form=bla_form, _extra_out=(kmap, s64))
    assert perturbation.LAST_FRAME_STATS["rebase_passes"] == 0
    fr, passes = oracle_pert_frame(m, arith=ARITH[arith],
                                   bla_eps=engine.ACCURATE_BLA_EPS if bla_form == "accurate" else None)
    assert passes == 0
    assert np.array_equal(it.view(np.uint32), fr.iter_map.view(np.uint32)), \
        int((it.view(np.uint32) != fr.iter_map.view(np.uint32)).sum())
    n_bad, max_diff = rgb_mismatch(rgb, fr.rgb)
    assert n_bad == 0, (n_bad, max_diff)
    if m["factor"] == 1:
        assert np.array_equal(kmap.cpu().numpy(), fr.kmap)


def test_one_pass_counters_count_rebases():
    """The coarse kernel's work counters: slot 3 holds each pixel's rebases."""
    import torch
    m = next(x for x in PMETA if x["name"] == "cfg3")
    re, im, rl = PS["cfg3__re"], PS["cfg3__im"], m["ref_len"]
    W, H = 96, 54
    L = _lib.load()
    d_re, d_im = torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda()
    po = torch.empty((rl + 1) * 6, dtype=torch.float64, device="cuda")
    _lib.check(L.ap_pack_orbit(C.c_void_p(d_re.data_ptr()), C.c_void_p(d_im.data_ptr()), rl,
                               C.c_void_p(po.data_ptr()), None), "ap_pack_orbit")
    it = torch.empty((H, W), dtype=torch.float32, device="cuda")
    cnt = torch.zeros((H, W, 4), dtype=torch.int32, device="cuda")
    p = abi.new_params(width=W, height=H, max_iter=20000, tier=abi.AP_TIER_PERTURB, arith=abi.AP_ARITH_REF_CPU,
                       dx_hi=m["dx"] * 20, dy_hi=m["dy"] * 20, ref_px=47.5, ref_py=26.5, ref_len=rl,
                       flags=abi.AP_FLAG_REBASE | abi.AP_FLAG_NO_RGB)
    b = abi.ApFrameBuffers()
    b.ref_re, b.ref_im = C.c_void_p(d_re.data_ptr()), C.c_void_p(d_im.data_ptr())
    b.iter_map = C.c_void_p(it.data_ptr())
    b.counters = C.c_void_p(cnt.data_ptr())
    b.orbit_packed = C.c_void_p(po.data_ptr())
    _lib.check(L.ap_render_pass(C.byref(p), C.byref(b), None), "ap_render_pass")
    c = cnt.cpu().numpy()
    assert c[..., 3].min() >= 0 and c[..., 3].mean() > 1.0  # most pixels restart more than once
    assert not c[..., 2].any()    # no direct-iteration stage
    assert np.all(c[..., 0] + c[..., 1] > 0)


def test_fast_profile_serves_one_pass_rebasing_only():
    """arith='fast' is the one-pass form's own arithmetic: other glitch modes and other
    passes refuse it."""
    with pytest.raises(ValueError):
        engine.render_frame_ssaa(64, 36, 1000, Decimal("-0.75"), Decimal("0.1"), Decimal("1e-14"), None,
                                 precision_mode="1e-300 (Perturbation)", glitch_mode="Pauldelbrot",
                                 arith="fast")
    import torch
    L = _lib.load()
    it = torch.zeros((8, 8), dtype=torch.float32, device="cuda")
    orbit = torch.zeros(5, dtype=torch.float64, device="cuda")
    p = abi.new_params(width=8, height=8, max_iter=10, tier=abi.AP_TIER_PERTURB, ref_len=4,
                       arith=abi.AP_ARITH_FAST, flags=abi.AP_FLAG_NO_RGB)
    b = abi.ApFrameBuffers()
    b.iter_map = C.c_void_p(it.data_ptr())
    b.ref_re = b.ref_im = C.c_void_p(orbit.data_ptr())
    assert L.ap_render_pass(C.byref(p), C.byref(b), None) == abi.AP_E_UNSUPPORTED


def test_one_pass_rejects_unserved_cases():
    with pytest.raises(NotImplementedError):
        engine.render_frame_ssaa(64, 36, 1000, Decimal("-0.79"), Decimal("0.27"), Decimal("1e-14"), None,
                                 precision_mode="1e-300 (Perturbation)", fractal_type=2, julia_cx=-0.8,
                                 julia_cy=0.156, glitch_mode=ONE_PASS_REBASING)
    with pytest.raises(NotImplementedError):
        engine.render_frame_ssaa(64, 36, 1000, Decimal("-0.75"), Decimal("0.1"), Decimal("1e-320"), None,
                                 precision_mode="1e-300 (Perturbation)", glitch_mode=ONE_PASS_REBASING)
    # the FP32 form rebases below 1e-300 at factor 1 only, and never Julia orbits
    with pytest.raises(NotImplementedError):
        engine.render_frame_ssaa(64, 36, 1000, Decimal("-0.75"), Decimal("0.1"), Decimal("1e-320"), None,
                                 ssaa_factor=2, precision_mode="1e-300 (Perturbation)",
                                 glitch_mode=ONE_PASS_REBASING, delta_form="fp32")
    with pytest.raises(NotImplementedError):
        engine.render_frame_ssaa(64, 36, 1000, Decimal("-0.79"), Decimal("0.27"), Decimal("1e-14"), None,
                                 precision_mode="1e-300 (Perturbation)", fractal_type=2, julia_cx=-0.8,
                                 julia_cy=0.156, glitch_mode=ONE_PASS_REBASING, delta_form="fp32")
    # the C-ABI refuses the flag outside the FP64-delta tier and for Julia orbits
    import torch
    L = _lib.load()
    p = abi.new_params(width=8, height=8, max_iter=10, tier=abi.AP_TIER_FLOATEXP, ref_len=4,
                       flags=abi.AP_FLAG_REBASE | abi.AP_FLAG_NO_RGB)
    it = torch.zeros((8, 8), dtype=torch.float32, device="cuda")
    orbit = torch.zeros(5, dtype=torch.float64, device="cuda")
    b = abi.ApFrameBuffers()
    b.iter_map = C.c_void_p(it.data_ptr())
    b.ref_re = b.ref_im = C.c_void_p(orbit.data_ptr())
    assert L.ap_render_pass(C.byref(p), C.byref(b), None) == abi.AP_E_UNSUPPORTED
    p.tier, p.fractal_type = abi.AP_TIER_PERTURB, 2
    assert L.ap_render_pass(C.byref(p), C.byref(b), None) == abi.AP_E_UNSUPPORTED
    p.fractal_type, p.ref_len = 0, 0
    assert L.ap_render_pass(C.byref(p), C.byref(b), None) == abi.AP_E_INVALID
