"""Whole perturbation-tier frames (orbit, BLA, passes, Pauldelbrot rebasing) through the
oracle against render_frame_cpu (math_core/engine.py:471) -- CPU only."""
import numpy as np
import pytest

from helpers import load_golden, oracle_pert_frame, rgb_mismatch

G, META = load_golden("render_pert.npz")

# The reference's histogram kernel (math_core/cpu_kernels.py:1887, fastmath) calls
# cpu_compute_perturbation_sample with float coordinates at factor 1 and with int64
# coordinates in its supersampling loop.  Numba compiles the int64 specialisation with
# the caller's fast-math flags (every floating-point operation of that copy is `fast`;
# the float copy has none), so its sums are reassociated and fused differently.  The
# samples it re-renders on rebase passes move slightly; those pixels are still flagged
# as glitched in the final map, and every other pixel is bit-exact.
FASTMATH_INLINED = {"cfg3_hist_ssaa2"}


@pytest.mark.parametrize("name", [m["name"] for m in META])
def test_pert_frame_matches_reference(name):
    m = next(x for x in META if x["name"] == name)
    fr, _ = oracle_pert_frame(m)
    ref_it = G[name + "__iter"]
    diff = fr.iter_map.view(np.uint32) != ref_it.view(np.uint32)
    if name in FASTMATH_INLINED:
        assert not np.any(diff & (fr.glitch_out == 0))
        assert diff.mean() < 0.02
        assert np.all(np.abs(fr.iter_map[diff] - ref_it[diff]) < 50.0)
    else:
        assert not diff.any(), int(diff.sum())
        n_bad, max_diff = rgb_mismatch(fr.rgb, G[name + "__rgb"])
        assert max_diff <= 1 and n_bad <= max(1, int(1e-4 * m["W"] * m["H"])), (n_bad, max_diff)
