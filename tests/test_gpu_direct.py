"""GPU parity of the direct tiers (FP64, double-double) through the engine's C ABI.

Each frame is rendered by fractura_b200.engine.render_frame_ssaa (the
reference's render entry point) and compared with
  * the reference's own output (golden fixtures): iteration maps bit-exact;
  * the oracle's restatement of the same passes: iteration maps, escape steps
    and RGB bit-exact, float64 smooth values within 1e-12 relative.
"""
from decimal import Decimal

import numpy as np
import pytest

from fractura_b200 import abi, engine
from helpers import load_golden, oracle_direct_frame, rgb_mismatch

pytestmark = pytest.mark.gpu


def gpu_frame(m, precision_mode, arith="ref_cpu"):
    import torch
    W, H = m["W"], m["H"]
    it = np.zeros((H, W), np.float32)
    kmap = torch.empty((H, W), dtype=torch.int32, device="cuda")
    s64 = torch.empty((H, W), dtype=torch.float64, device="cuda")
    rgb = engine.render_frame_ssaa(
        W, H, m["max_iter"], Decimal(m["cx"]), Decimal(m["cy"]), Decimal(m["width"]), None,
        ssaa_factor=m["factor"], edge_threshold=0.35, color_scheme_id=m["scheme"],
        precision_mode=precision_mode, fractal_type=m["fractal_type"], julia_cx=m["julia_cx"],
        julia_cy=m["julia_cy"], gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"],
        palette_offset=m["offset"], color_density=m["density"], color_contrast=m["contrast"],
        h_iter_buf=it, arith=arith, _extra_out=(kmap, s64))
    return rgb, it, kmap.cpu().numpy(), s64.cpu().numpy()


def check_against_oracle(m, tier, arith_name, arith_code):
    rgb, it, kmap, s64 = gpu_frame(m, "1e-24 (DD)" if tier == abi.AP_TIER_DD else "1e-12 (FP64)",
                                   arith_name)
    fr = oracle_direct_frame(m, tier=tier, arith=arith_code)
    assert np.array_equal(it.view(np.uint32), fr.iter_map.view(np.uint32))
    assert np.array_equal(kmap, fr.kmap)
    esc = fr.s64 >= 0
    assert np.all(np.abs(s64[esc] - fr.s64[esc]) <= 1e-12 * np.abs(fr.s64[esc]))
    n_bad, max_diff = rgb_mismatch(rgb, fr.rgb)
    assert n_bad == 0, (n_bad, max_diff)
    return rgb, it


FP64_CASES = ["cfg1_hist", "cfg1_s0", "ssaa2_s0", "ssaa2_hist", "ssaa3_julia", "scheme1", "scheme2",
              "scheme3", "scheme4", "scheme5", "scheme6", "scheme7", "scheme8", "scheme9",
              "scheme10", "ship_s2", "multibrot_s5", "shipjulia_hist"]


@pytest.mark.parametrize("case", FP64_CASES)
def test_fp64_frame_matches_reference_and_oracle(case):
    g, meta = load_golden("render_fp64.npz")
    m = next(x for x in meta if x["name"] == case)
    rgb, it = check_against_oracle(m, abi.AP_TIER_FP64, "ref_cpu", abi.AP_ARITH_REF_CPU)
    assert np.array_equal(it.view(np.uint32), g[case + "__iter"].view(np.uint32))
    n_bad, max_diff = rgb_mismatch(rgb, g[case + "__rgb"])
    assert max_diff <= 1 and n_bad <= max(1, int(1e-4 * m["W"] * m["H"]))


@pytest.mark.parametrize("case", ["cfg1_s0", "ssaa2_hist", "ship_s2", "multibrot_s5"])
def test_fp64_cuda_profile_matches_oracle(case):
    _, meta = load_golden("render_fp64.npz")
    m = next(x for x in meta if x["name"] == case)
    check_against_oracle(m, abi.AP_TIER_FP64, "ref_cuda", abi.AP_ARITH_REF_CUDA)


DD_CASES = ["cfg2_quarter", "cfg2_hist", "dd_mandel", "dd_mandel_ssaa", "dd_julia", "dd_shipjulia",
            "dd_multibrot3", "dd_multibrot5"]


@pytest.mark.parametrize("case", DD_CASES)
def test_dd_frame_matches_reference_and_oracle(case):
    g, meta = load_golden("render_dd.npz")
    m = next(x for x in meta if x["name"] == case)
    rgb, it = check_against_oracle(m, abi.AP_TIER_DD, "ref_cpu", abi.AP_ARITH_REF_CPU)
    assert np.array_equal(it.view(np.uint32), g[case + "__iter"].view(np.uint32))


@pytest.mark.parametrize("case", ["cfg2_quarter", "dd_mandel", "dd_multibrot3"])
def test_dd_cuda_profile_matches_oracle(case):
    _, meta = load_golden("render_dd.npz")
    m = next(x for x in meta if x["name"] == case)
    check_against_oracle(m, abi.AP_TIER_DD, "ref_cuda", abi.AP_ARITH_REF_CUDA)


def test_recolor_frame_matches_fresh_render():
    """recolor_frame (math_core/engine.py:2138) reproduces a render's colours from its iter map."""
    import torch
    from fractura_b200.config import RenderParameters
    _, meta = load_golden("render_fp64.npz")
    m = next(x for x in meta if x["name"] == "scheme7")
    W, H = m["W"], m["H"]
    d_iter = torch.empty((H, W), dtype=torch.float32, device="cuda")
    for scheme in (7, 11):
        q = RenderParameters(target_w=W, target_h=H, max_iter=m["max_iter"],
                             center_x_dec=Decimal(m["cx"]), center_y_dec=Decimal(m["cy"]),
                             plot_width_dec=Decimal(m["width"]), cmap_name=None,
                             color_scheme_id=scheme, precision_mode="1e-12 (FP64)",
                             palette_offset=0.2, d_iter_buf=d_iter)
        rgb = engine.render_frame(q)
        again = engine.recolor_frame(q, d_iter_buf=d_iter)
        assert np.array_equal(rgb, again)


def test_hdr_output_is_uint16():
    _, meta = load_golden("render_fp64.npz")
    m = next(x for x in meta if x["name"] == "scheme5")
    rgb = engine.render_frame_ssaa(m["W"], m["H"], m["max_iter"], Decimal(m["cx"]), Decimal(m["cy"]),
                                   Decimal(m["width"]), None, color_scheme_id=5,
                                   precision_mode="1e-12 (FP64)", is_hdr=True)
    assert rgb.dtype == np.uint16 and rgb.max() > 255
