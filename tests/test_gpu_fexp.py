"""GPU parity of the FloatExp tier (views below 1e-300).

  * one render pass on the device equals the oracle's pass value for value
    (smooth float32, float64, escape step, glitch flag), both arithmetic
    profiles, with and without chained BLA, on crops of the golden views;
  * a whole frame through the engine (FloatExp tier, Pauldelbrot rebasing)
    equals the oracle's frame.
"""
import ctypes as C
from decimal import Decimal

import numpy as np
import pytest

import oracle
from fractura_b200 import _lib, abi, engine
from fractura_b200 import high_precision as hp
from fractura_b200.palette import synthetic_lut
from helpers import load_golden, oracle_pert_frame, rgb_mismatch
from test_oracle_fexp import floatexp_params

pytestmark = pytest.mark.gpu

G, META = load_golden("fexp_samples.npz")
CASES = [m["name"] for m in META]
CROP_W, CROP_H = 160, 90


def _device_pass(p, re, im, T):
    import torch
    H, W = p.height, p.width
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    d = dict(re=t(re), im=t(im), lut=t(synthetic_lut()))
    if T is not None:
        d["bla"] = t(T)
    out = dict(iter=torch.zeros((H, W), dtype=torch.float32, device="cuda"),
               kmap=torch.zeros((H, W), dtype=torch.int32, device="cuda"),
               s64=torch.zeros((H, W), dtype=torch.float64, device="cuda"),
               glitch=torch.zeros((H, W), dtype=torch.uint8, device="cuda"),
               gin=torch.zeros((H, W), dtype=torch.uint8, device="cuda"),
               rgb=torch.zeros((H, W, 3), dtype=torch.uint8, device="cuda"))
    b = abi.ApFrameBuffers()
    ptr = lambda x: C.c_void_p(x.data_ptr())
    b.ref_re, b.ref_im, b.lut = ptr(d["re"]), ptr(d["im"]), ptr(d["lut"])
    b.bla = ptr(d["bla"]) if T is not None else None
    b.iter_map, b.kmap, b.s64 = ptr(out["iter"]), ptr(out["kmap"]), ptr(out["s64"])
    b.glitch_out, b.glitch_in, b.rgb = ptr(out["glitch"]), ptr(out["gin"]), ptr(out["rgb"])
    L = _lib.load()
    _lib.check(L.ap_render_pass(C.byref(p), C.byref(b), None), "ap_render_pass")
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in out.items()}


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("variant", ["plain", "bla"])
@pytest.mark.parametrize("arith", [abi.AP_ARITH_REF_CPU, abi.AP_ARITH_REF_CUDA])
def test_floatexp_pass_matches_oracle(name, variant, arith):
    m = next(x for x in META if x["name"] == name)
    re, im = G[name + "__re"], G[name + "__im"]
    use_bla, p = floatexp_params(m, variant, arith)
    p.width, p.height = min(m["W"], CROP_W), min(m["H"], CROP_H)
    p.mode = abi.AP_MODE_COARSE
    T = oracle.build_bla(re, im, m["ref_len"], m["fractal_type"], 1e-6, 16, m["gen_n"], m["gen_kr"],
                         m["gen_ki"]) if use_bla else None
    got = _device_pass(p, re, im, T)
    fr = oracle.Frame(p.width, p.height, lut=synthetic_lut())
    fr.ref_re, fr.ref_im, fr.bla = np.ascontiguousarray(re), np.ascontiguousarray(im), T
    oracle.render_pass(p, fr)
    assert np.array_equal(got["iter"].view(np.uint32), fr.iter_map.view(np.uint32)), \
        int((got["iter"].view(np.uint32) != fr.iter_map.view(np.uint32)).sum())
    assert np.array_equal(got["kmap"], fr.kmap)
    assert np.array_equal(got["s64"].view(np.uint64), fr.s64.view(np.uint64))
    assert np.array_equal(got["glitch"], fr.glitch_out)
    assert np.array_equal(got["rgb"], fr.rgb)


@pytest.mark.parametrize("name", ["fexp_mandel", "fexp_ship", "fexp_julia", "fexp_multibrot3"])
@pytest.mark.parametrize("arith", ["ref_cpu", "ref_cuda"])
def test_floatexp_frame_through_engine(name, arith):
    m = next(x for x in META if x["name"] == name)
    W, H = 160, 90
    mm = dict(m, W=W, H=H, factor=1, scheme=0, bbsa_order=32, glitch_mode="Pauldelbrot")
    hp.clear_reference_orbit_cache()
    it = np.zeros((H, W), np.float32)
    rgb = engine.render_frame_ssaa(
        W, H, m["max_iter"], Decimal(m["cx"]), Decimal(m["cy"]), Decimal(m["width"]), None,
        color_scheme_id=0, precision_mode="1e-300 (Perturbation)", fractal_type=m["fractal_type"],
        julia_cx=m["julia_cx"], julia_cy=m["julia_cy"], bbsa_tol=1e-6, bbsa_order=32,
        glitch_mode="Pauldelbrot", gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"],
        h_iter_buf=it, arith=arith)
    fr, _ = oracle_pert_frame(mm, arith=0 if arith == "ref_cpu" else 1)
    assert np.mean(it >= 0) > 0.5
    assert np.array_equal(it.view(np.uint32), fr.iter_map.view(np.uint32)), \
        int((it.view(np.uint32) != fr.iter_map.view(np.uint32)).sum())
    n_bad, max_diff = rgb_mismatch(rgb, fr.rgb)
    assert n_bad == 0, (n_bad, max_diff)
