"""Precision of the engine's delta and BLA forms at the 1e-160 view of config 3.

The ground truth (tests/golden/truth_cfg3.npz) is direct z^2 + c iteration in
700-bit arithmetic on a 64 x 64 subsample (every 30th column, every 17th row)
of the 1920 x 1080 frame.  Smooth errors are absolute, on the float64 smooth
value s64 = (k + 1) - nu.  Frames here use one reference (glitch mode off), so
that the arithmetic is compared and not the rebase loop's choice of references.
"""
import ctypes as C
import json
import os
from decimal import Decimal

import numpy as np
import pytest

import oracle
from fractura_b200 import _lib, engine
from fractura_b200 import high_precision as hp
from fractura_b200.config import ACCURATE_BLA_EPS
from helpers import GOLDEN, load_golden, oracle_pert_frame, rgb_mismatch

pytestmark = pytest.mark.gpu

PS, PMETA = load_golden("pert_samples.npz")
RS, RMETA = load_golden("render_pert.npz")


def _truth():
    t = np.load(os.path.join(GOLDEN, "truth_cfg3.npz"))
    return t["s"], t["rows"], t["cols"]


@pytest.mark.parametrize("dc_max", [0.0, 1e-12, 3e-3])
@pytest.mark.parametrize("name", [m["name"] for m in PMETA if m["bla_shape"][0] > 1])
def test_device_bla_dc_table_matches_oracle(name, dc_max):
    import torch
    m = next(x for x in PMETA if x["name"] == name)
    re, im = PS[name + "__re"], PS[name + "__im"]
    rl = m["ref_len"]
    d_re, d_im = torch.from_numpy(re).cuda(), torch.from_numpy(im).cuda()
    out = torch.empty((16, rl, 5), dtype=torch.float64, device="cuda")
    L = _lib.load()
    _lib.check(L.ap_build_bla_dc(C.c_void_p(d_re.data_ptr()), C.c_void_p(d_im.data_ptr()), rl,
                                 m["fractal_type"], ACCURATE_BLA_EPS, dc_max, 16, m["gen_n"],
                                 m["gen_kr"], m["gen_ki"], C.c_void_p(out.data_ptr()), None),
               "ap_build_bla_dc")
    T = oracle.build_bla_dc(re, im, rl, m["fractal_type"], ACCURATE_BLA_EPS, dc_max, 16, m["gen_n"],
                            m["gen_kr"], m["gen_ki"])
    got = out.cpu().numpy()
    if m["fractal_type"] == 4 and m["gen_n"] > 3:
        # level 0 goes through pow(); CUDA's and glibc's pow may differ by an ulp
        assert np.allclose(got, T, rtol=1e-13, atol=0)
    else:
        assert got.tobytes() == T.tobytes()
    # radii never increase with the level (the level search relies on it)
    R = got[:, :, 4]
    assert np.all(np.diff(R, axis=0) <= 0)


@pytest.mark.parametrize("name", ["cfg3_bla_pauldelbrot", "cfg3_hist", "cfg3_ssaa2"])
def test_accurate_bla_frame_matches_oracle(name):
    """bla_form="accurate" through the engine (rebasing included) equals the oracle's
    frame with the dc-aware tables, value for value."""
    m = next(x for x in RMETA if x["name"] == name)
    W, H = m["W"], m["H"]
    hp.clear_reference_orbit_cache()
    it = np.zeros((H, W), np.float32)
    rgb = engine.render_frame_ssaa(
        W, H, m["max_iter"], Decimal(m["cx"]), Decimal(m["cy"]), Decimal(m["width"]), None,
        ssaa_factor=m["factor"], color_scheme_id=m["scheme"], precision_mode="1e-300 (Perturbation)",
        fractal_type=m["fractal_type"], bbsa_tol=1e-6, bbsa_order=32, glitch_mode=m["glitch_mode"],
        h_iter_buf=it, arith="ref_cpu", bla_form="accurate")
    mm = dict(m, bbsa_order=32)
    fr, _ = oracle_pert_frame(mm, bla_eps=ACCURATE_BLA_EPS)
    assert np.array_equal(it.view(np.uint32), fr.iter_map.view(np.uint32)), \
        int((it.view(np.uint32) != fr.iter_map.view(np.uint32)).sum())
    n_bad, max_diff = rgb_mismatch(rgb, fr.rgb)
    assert n_bad == 0, (n_bad, max_diff)


def _cfg3_single_ref(**over):
    import torch
    with open(os.path.join(GOLDEN, "workloads.json")) as f:
        cx, cy = json.load(f)["config3_centre"]
    W, H = 1920, 1080
    kmap = torch.empty((H, W), dtype=torch.int32, device="cuda")
    s64 = torch.empty((H, W), dtype=torch.float64, device="cuda")
    hp.clear_reference_orbit_cache()
    kw = dict(bbsa_tol=1e-6, bbsa_order=32, glitch_mode="Off (Single-Ref)", arith="ref_cpu")
    kw.update(over)
    engine.render_frame_ssaa(W, H, 20000, Decimal(cx), Decimal(cy), Decimal("1e-160"), None,
                             color_scheme_id=0, precision_mode="1e-300 (Perturbation)",
                             fractal_type=0, _extra_out=(kmap, s64), **kw)
    torch.cuda.synchronize()
    return kmap.cpu().numpy(), s64.cpu().numpy()


def _errors(k, s64):
    truth, rows, cols = _truth()
    ks, ss = k[np.ix_(rows, cols)], s64[np.ix_(rows, cols)]
    err = np.abs(ss - truth)
    return err, float(np.mean(ks == np.floor(truth)))


def test_config3_plain_fp64_against_truth():
    k, s = _cfg3_single_ref(bbsa_order=0)
    err, k_match = _errors(k, s)
    assert k_match >= 0.999, k_match
    assert np.percentile(err, 99) <= 1e-4, np.percentile(err, 99)


def test_config3_accurate_bla_against_truth_and_plain():
    k0, s0 = _cfg3_single_ref(bbsa_order=0)
    k1, s1 = _cfg3_single_ref(bla_form="accurate")
    err, k_match = _errors(k1, s1)
    assert k_match >= 0.999, k_match
    assert np.percentile(err, 99) <= 1e-4, np.percentile(err, 99)
    # against the plain FP64-delta frame: identical escape steps on >= 99.9 % of pixels
    same_k = float(np.mean(k0 == k1))
    assert same_k >= 0.999, same_k
    assert np.percentile(np.abs(s1 - s0), 99.9) <= 1e-4
