"""The FP32-mantissa FloatExp form (AP_TIER_FLOATEXP32, fe32_coarse_kernel, ap_pack_fe32).

* Packing: the FP32 orbit copy holds each Z rounded to float and the close-approach
  marks; every BLA entry's (mantissa, exponent) pairs give back the FP64 coefficient to
  float precision; the radius rows are r^2 2^600.
* Width 1e-1000 (config 3b, 1920x1080): the FP64-mantissa FloatExp frame (same BLA
  form) is reproduced: identical escape steps and smooth values within 1e-4 (the whole
  view escapes in a few leaps, so 24-bit deltas carry it); the reference's own FloatExp
  samples (fexp_samples.npz) agree on the escape step.
* Width 1e-160 (config 3, 1920x1080): the error against the 700-bit ground truth stays at
  the level this form is documented at -- it cannot meet the 1e-4 bound there: the view's
  values need about 40 bits of delta precision (a one-ulp change of dc in float32 alone
  moves p99 by 0.47) -- and the test guards that level against regressions.
"""
import ctypes as C
from decimal import Decimal

import numpy as np
import pytest

from fractura_b200 import _lib, engine
from fractura_b200 import high_precision as hp
from helpers import GOLDEN, load_golden

pytestmark = pytest.mark.gpu

FG, FMETA = load_golden("fexp_samples.npz")
PS, PMETA = load_golden("pert_samples.npz")


def _fe32_frame(m, width, max_iter, glitch_mode, W=1920, H=1080):
    import torch
    kmap = torch.empty((H, W), dtype=torch.int32, device="cuda")
    s64 = torch.empty((H, W), dtype=torch.float64, device="cuda")
    it = np.zeros((H, W), np.float32)
    hp.clear_reference_orbit_cache()
    engine.render_frame_ssaa(W, H, max_iter, Decimal(m["cx"]), Decimal(m["cy"]), Decimal(width), None,
                             precision_mode="1e-300 (Perturbation)", bbsa_order=32, bbsa_tol=1e-6,
                             glitch_mode=glitch_mode, arith="ref_cuda", bla_form="accurate",
                             delta_form="fp32", h_iter_buf=it, _extra_out=(kmap, s64))
    return it, kmap.cpu().numpy(), s64.cpu().numpy()


def test_pack_fe32_records():
    import torch
    m = next(x for x in PMETA if x["name"] == "cfg3")
    re, im, rl = PS["cfg3__re"], PS["cfg3__im"], m["ref_len"]
    import oracle
    T = oracle.build_bla_dc(re, im, rl, 0, 1e-14, 1e-157, 16, 3, 0.25, 1.0)
    L = _lib.load()
    d_re, d_im, d_T = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (re, im, T))
    po = torch.empty(6 * (rl + 1), dtype=torch.float64, device="cuda")
    ptr = lambda t: C.c_void_p(t.data_ptr())
    _lib.check(L.ap_pack_orbit(ptr(d_re), ptr(d_im), rl, ptr(po), None), "ap_pack_orbit")
    pf = torch.empty(80 * rl, dtype=torch.float64, device="cuda")
    _lib.check(L.ap_pack_fe32(ptr(po), rl, ptr(d_T), 16, ptr(po[4 * (rl + 1):]), ptr(pf), None), "ap_pack_fe32")
    orb32 = po[4 * (rl + 1):].cpu().numpy().view(np.float32).reshape(rl + 1, 4)
    assert np.array_equal(orb32[:, 0], re.astype(np.float32))
    assert np.array_equal(orb32[:, 1], im.astype(np.float32))
    r2 = re * re + im * im
    assert np.array_equal(orb32[:, 3] != 0, r2 < 2.0 ** -100)    # close approaches take the FP64 path
    raw = pf.cpu().numpy()
    Rs = raw[:16 * rl].reshape(rl, 16)
    assert np.array_equal(Rs, np.ldexp(T[:, :, 4].T, 600))
    rec = raw[16 * rl:].view(np.uint8).reshape(rl, 16, 32)
    mant = rec[..., :16].copy().view(np.float32).reshape(rl, 16, 4)
    ex = rec[..., 16:24].copy().view(np.int32).reshape(rl, 16, 2)
    for comp, (re_i, im_i, e_i) in enumerate(((0, 1, 0), (2, 3, 1))):   # A, then B
        got_r = np.ldexp(mant[..., re_i].astype(np.float64), ex[..., e_i])
        got_i = np.ldexp(mant[..., im_i].astype(np.float64), ex[..., e_i])
        want_r = np.transpose(T[:, :, 2 * comp], (1, 0))
        want_i = np.transpose(T[:, :, 2 * comp + 1], (1, 0))
        scale = np.maximum(np.abs(want_r), np.abs(want_i))
        ok = scale > 1e-300
        # the pair shares one exponent: each component is exact to a float ulp of the larger
        assert np.all(np.abs(got_r - want_r)[ok] <= 2.0 ** -23 * scale[ok])
        assert np.all(np.abs(got_i - want_i)[ok] <= 2.0 ** -23 * scale[ok])


def _fp64_floatexp_frame(m, W, H):
    import torch
    kmap = torch.empty((H, W), dtype=torch.int32, device="cuda")
    s64 = torch.empty((H, W), dtype=torch.float64, device="cuda")
    hp.clear_reference_orbit_cache()
    engine.render_frame_ssaa(W, H, m["max_iter"], Decimal(m["cx"]), Decimal(m["cy"]), Decimal(m["width"]), None,
                             precision_mode="1e-300 (Perturbation)", bbsa_order=32, bbsa_tol=1e-6,
                             glitch_mode="Off (Single-Ref)", arith="ref_cuda", bla_form="accurate",
                             _extra_out=(kmap, s64))
    return kmap.cpu().numpy(), s64.cpu().numpy()


def test_fe32_at_1e1000_matches_the_fp64_floatexp_frame():
    """At 1e-1000 the FP32 form reproduces the FP64-mantissa FloatExp frame (same BLA form):
    identical escape steps on every pixel, smooth values within 1e-4; and the reference's
    own FloatExp samples (its BLA table) agree on the escape step."""
    m = next(x for x in FMETA if x["name"] == "fexp_cfg3")
    W, H = m["W"], m["H"]
    it, k, s64 = _fe32_frame(m, m["width"], m["max_iter"], "Off (Single-Ref)", W, H)
    k64, s64_64 = _fp64_floatexp_frame(m, W, H)
    assert np.array_equal(k, k64)
    esc = k64 >= 0
    assert np.max(np.abs(s64[esc] - s64_64[esc])) <= 1e-4
    st = m["stride"]
    want = FG["fexp_cfg3__bla_s"]
    got = it[::st, ::st][:want.shape[0], :want.shape[1]]
    assert np.mean(np.floor(got) == np.floor(want)) >= 0.99


@pytest.mark.parametrize("glitch_mode", ["Off (Single-Ref)", "Pauldelbrot"])
def test_fe32_at_1e160_error_level(glitch_mode):
    m = next(x for x in PMETA if x["name"] == "cfg3")
    t = np.load(f"{GOLDEN}/truth_cfg3.npz")
    truth, rows, cols = t["s"], t["rows"], t["cols"]
    _, k, s64 = _fe32_frame(m, m["width"], 200000, glitch_mode)
    err = np.abs(s64[np.ix_(rows, cols)] - truth)
    kid = float(np.mean(k[np.ix_(rows, cols)] == np.floor(truth)))
    p99 = float(np.percentile(err, 99))
    # the documented level of the FP32 form at this view (p99 about 1.8-6, identical k 97-98 %)
    assert p99 <= 10.0 and kid >= 0.95, (p99, kid)
    assert float(np.median(err)) <= 1e-3, float(np.median(err))
