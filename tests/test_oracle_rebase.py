"""One-pass rebasing (AP_FLAG_REBASE) in the oracle, against the 700-bit ground truth.

The reference has no one-pass mode: its Pauldelbrot loop re-renders glitched pixels
around new references (math_core/engine.py:1890-2113).  The engine's extension
restarts each pixel's delta from the orbit's start when |z| < |dz| or the reference
ends.  Its accuracy is pinned at the config-3 view (1920x1080 at width 1e-160,
max_iter 200000) by tests/golden/truth_cfg3.npz, on the reference's own orbit
(pert_samples.npz, cfg3).  Bound: smooth-value error p99 <= 1e-4 and an identical
escape step on >= 99.9 % of the 64 x 64 samples.
"""
import os

import numpy as np
import pytest

import oracle
from fractura_b200 import abi
from fractura_b200.perturbation import max_delta_c
from helpers import GOLDEN, load_golden

PS, PMETA = load_golden("pert_samples.npz")

P99_BOUND = 1e-4
K_IDENTICAL_BOUND = 0.999


def truth():
    t = np.load(os.path.join(GOLDEN, "truth_cfg3.npz"))
    return t["s"], t["rows"], t["cols"]


def cfg3_params(arith, bla, flags=abi.AP_FLAG_REBASE):
    m = next(x for x in PMETA if x["name"] == "cfg3")
    re, im, rl = PS["cfg3__re"], PS["cfg3__im"], m["ref_len"]
    T = None
    if bla:
        dcm = max_delta_c(m["ref_px"], m["ref_py"], m["W"], m["H"], m["dx"], m["dy"])
        T = oracle.build_bla_dc(re, im, rl, 0, 1e-14, dcm, 16, 3, 0.25, 1.0)
    p = abi.new_params(width=m["W"], height=m["H"], max_iter=m["max_iter"], tier=abi.AP_TIER_PERTURB,
                       arith=arith, dx_hi=m["dx"], dy_hi=m["dy"], ref_px=m["ref_px"], ref_py=m["ref_py"],
                       ref_cx=float(m["ref_cx"]), ref_cy=float(m["ref_cy"]), ref_len=rl,
                       bla_levels=16 if T is not None else 0, flags=flags)
    return p, re, im, T


def errors(k, s64, ts):
    err = np.abs(s64 - ts)
    return float(np.percentile(err, 99)), float(np.mean(k == np.floor(ts))), float(err.max())


@pytest.mark.parametrize("arith", [abi.AP_ARITH_REF_CPU, abi.AP_ARITH_REF_CUDA, abi.AP_ARITH_FAST])
@pytest.mark.parametrize("bla", [True, False])
def test_one_pass_config3_meets_accuracy_bound(arith, bla):
    ts, rows, cols = truth()
    p, re, im, T = cfg3_params(arith, bla)
    _, g, k, s64 = oracle.pert_grid(p, re, im, T, cols.astype(np.float64), rows.astype(np.float64),
                                    with_s64=True)
    p99, kid, mx = errors(k, s64, ts)
    assert not g.any()  # no pixel is left glitched: every one is served in the single pass
    assert p99 <= P99_BOUND, (p99, kid, mx)
    assert kid >= K_IDENTICAL_BOUND, (p99, kid, mx)


def test_single_reference_pauldelbrot_flags_samples_the_one_pass_form_serves():
    """The same view on one reference with the reference's Pauldelbrot test: samples that
    outlive the reference (ref_len 8050 < max_iter) are flagged glitched, and the
    reference would re-render them around new references.  The one-pass form serves
    them in the same pass (test above: none flagged, bound met)."""
    ts, rows, cols = truth()
    p, re, im, T = cfg3_params(abi.AP_ARITH_REF_CPU, True, flags=abi.AP_FLAG_NAN_GUARD)
    p.strict_glitch = 1
    _, g, k, _ = oracle.pert_grid(p, re, im, T, cols.astype(np.float64), rows.astype(np.float64),
                                  with_s64=True)
    assert g.sum() >= 10
    assert np.all(k[g > 0] >= p.ref_len)


def test_one_pass_render_pass_equals_sample_grid():
    """The oracle's render pass takes the same rebase sample as its sample grid."""
    m = next(x for x in PMETA if x["name"] == "cfg3")
    p, re, im, T = cfg3_params(abi.AP_ARITH_REF_CPU, True)
    W, H = 48, 27
    p.width, p.height, p.max_iter = W, H, 20000
    p.dx_hi, p.dy_hi = m["dx"] * 40, m["dy"] * 40
    p.ref_px, p.ref_py = 23.5, 13.5
    p.flags |= abi.AP_FLAG_NO_RGB
    fr = oracle.Frame(W, H)
    fr.ref_re, fr.ref_im, fr.bla = re, im, T
    oracle.render_pass(p, fr)
    s, g, k = oracle.pert_grid(p, re, im, T, np.arange(W, dtype=np.float64), np.arange(H, dtype=np.float64))
    assert np.array_equal(fr.iter_map.view(np.uint32), s.view(np.uint32))
    assert not g.any() and not fr.glitch_out.any()


@pytest.mark.parametrize("name", ["ship", "multibrot3", "multibrot4"])
def test_one_pass_other_formulas(name):
    """Burning Ship and Multibrot views (chaotic: no ground truth there): every sample
    ends without a glitch flag, and a sample that escapes before its first rebase equals
    the single-reference value bit for bit.  A rebase needs |Z_m + dz| < |dz|, which
    |dz| < |Z_m| / 2 rules out; the single-reference run's samples that escape while
    every |dz| stayed below that bound are therefore the ones to compare."""
    m = next(x for x in PMETA if x["name"] == name)
    re, im, rl = PS[name + "__re"], PS[name + "__im"], m["ref_len"]
    kw = dict(width=m["W"], height=m["H"], max_iter=m["max_iter"], tier=abi.AP_TIER_PERTURB,
              arith=abi.AP_ARITH_REF_CPU, fractal_type=m["fractal_type"], gen_n=m["gen_n"],
              gen_kr=m["gen_kr"], gen_ki=m["gen_ki"], dx_hi=m["dx"], dy_hi=m["dy"],
              ref_px=m["ref_px"], ref_py=m["ref_py"], ref_len=rl)
    st = m["stride"]
    xs = np.arange(0, m["W"], st, dtype=np.float64)
    ys = np.arange(0, m["H"], st, dtype=np.float64)
    s, g, k = oracle.pert_grid(abi.new_params(flags=abi.AP_FLAG_REBASE, **kw), re, im, None, xs, ys)
    assert not g.any()
    assert np.all((k >= 0) | (k == -1))
    s1, _, k1 = oracle.pert_grid(abi.new_params(flags=0, **kw), re, im, None, xs, ys)
    same = s.view(np.uint32) == s1.view(np.uint32)
    # wherever the two differ, a rebase happened: never before the reference first comes
    # within reach of zero in delta terms, so at least the earliest escapes agree
    first = int(np.min(k1[k1 >= 0]))
    assert np.all(same[k1 == first])
    assert same.mean() > 0.05
