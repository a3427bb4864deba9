"""The oracle against vectors produced by running the reference (CPU only)."""
import numpy as np
import pytest

import oracle
from fractura_b200 import abi
from helpers import load_golden, oracle_direct_frame, rgb_mismatch


def test_fp64_samples_bit_exact():
    """cpu_compute_fp64_sample (math_core/cpu_kernels.py:228) on all five formulas."""
    g, meta = load_golden("fp64_samples.npz")
    for m in meta:
        p = abi.new_params(fractal_type=m["fractal_type"], max_iter=m["max_iter"],
                           arith=abi.AP_ARITH_REF_CPU, julia_cx_hi=m["julia_cx"],
                           julia_cy_hi=m["julia_cy"], gen_n=m["gen_n"], gen_kr=m["gen_kr"],
                           gen_ki=m["gen_ki"])
        s32, s64, k = oracle.fp64_grid(p, g[m["name"] + "__x"], g[m["name"] + "__y"])
        ref = g[m["name"] + "__s"]
        assert np.array_equal(s32.view(np.uint32), ref.view(np.uint32)), m["name"]
        esc = ref >= 0
        # float64 smooth value agrees with the float32 one to float32 rounding
        assert np.all(np.abs(s64[esc] - ref[esc]) <= np.abs(ref[esc]) * 2e-7 + 1e-6)
        assert np.all(k[~esc] < 0) and np.all(k[esc] >= 0)


def test_fp64_cuda_profile_boundary_fraction():
    """The CUDA-source profile differs from the compiled CPU reference only on boundary samples."""
    g, meta = load_golden("fp64_samples.npz")
    total = changed = 0
    for m in meta:
        p = abi.new_params(fractal_type=m["fractal_type"], max_iter=m["max_iter"],
                           arith=abi.AP_ARITH_REF_CUDA, julia_cx_hi=m["julia_cx"],
                           julia_cy_hi=m["julia_cy"], gen_n=m["gen_n"], gen_kr=m["gen_kr"],
                           gen_ki=m["gen_ki"])
        s32, _, _ = oracle.fp64_grid(p, g[m["name"] + "__x"], g[m["name"] + "__y"])
        ref = g[m["name"] + "__s"]
        changed += int((np.floor(s32) != np.floor(ref)).sum())
        total += ref.size
    # boundary-rich zooms: a few percent of samples change escape step under contraction
    assert changed / total < 0.05


@pytest.mark.parametrize("case", ["cfg1_hist", "cfg1_s0", "ssaa2_s0", "ssaa2_hist", "ssaa3_julia",
                                  "scheme1", "scheme2", "scheme3", "scheme4", "scheme5", "scheme6",
                                  "scheme7", "scheme8", "scheme9", "scheme10", "ship_s2",
                                  "multibrot_s5", "shipjulia_hist"])
def test_fp64_frames_match_reference(case):
    """render_frame_cpu (math_core/engine.py:471) frames: iteration maps bit-exact; RGB within
    one level on at most 1e-4 of pixels (the reference's CPU colour is fastmath-compiled)."""
    g, meta = load_golden("render_fp64.npz")
    m = next(x for x in meta if x["name"] == case)
    fr = oracle_direct_frame(m)
    assert np.array_equal(fr.iter_map.view(np.uint32), g[case + "__iter"].view(np.uint32))
    n_bad, max_diff = rgb_mismatch(fr.rgb, g[case + "__rgb"])
    assert max_diff <= 1
    assert n_bad <= max(1, int(1e-4 * m["W"] * m["H"])), (n_bad, max_diff)


@pytest.mark.parametrize("case", ["cfg2_quarter", "cfg2_hist", "dd_mandel", "dd_mandel_ssaa",
                                  "dd_julia", "dd_shipjulia", "dd_multibrot3", "dd_multibrot5"])
def test_dd_frames_match_reference(case):
    """Double-double frames (math_core/cpu_kernels.py:1220 cpu_render_dd_kernel): iteration maps
    bit-exact; RGB within one level on at most 1e-4 of pixels."""
    g, meta = load_golden("render_dd.npz")
    m = next(x for x in meta if x["name"] == case)
    fr = oracle_direct_frame(m, tier=abi.AP_TIER_DD)
    assert np.array_equal(fr.iter_map.view(np.uint32), g[case + "__iter"].view(np.uint32))
    n_bad, max_diff = rgb_mismatch(fr.rgb, g[case + "__rgb"])
    assert max_diff <= 1
    assert n_bad <= max(1, int(1e-4 * m["W"] * m["H"])), (n_bad, max_diff)
