"""Adaptive max-iter probe through the oracle against the reference's CPU probe -- CPU only.

The probe (math_core/engine.py:1063-1281) renders a small grid whose corners are pixel
centres, one sample per pixel with the plain (non-BLA) sample, searching to
max(1000, 2 base_iter); the depth is max(1.35 p98, 1.2 max) of the escaped values
(:1051-1060).  The fixtures are the reference's probe maps, recorded where its CPU
branch hands them to get_adaptive_max_iter_from_probe, and the depths it returned
(tests/golden/make_golden.py, section probe)."""
import numpy as np
import pytest

from fractura_b200 import abi, engine
from helpers import load_golden, oracle_probe, probe_search

G, META = load_golden("probe.npz")


@pytest.mark.parametrize("name", [m["name"] for m in META])
def test_probe_map_matches_reference(name):
    m = next(x for x in META if x["name"] == name)
    it = oracle_probe(m)
    want = G[name + "__iter"]
    diff = it.view(np.uint32) != want.view(np.uint32)
    assert not diff.any(), int(diff.sum())
    assert engine.get_adaptive_max_iter_from_probe(it, m["base_iter"]) == m["depth"]


def test_probe_fixtures_cover_every_tier_and_formula():
    tiers = {engine.select_tier(__import__("decimal").Decimal(m["width"]), m["precision_mode"]) for m in META}
    assert tiers == {abi.AP_TIER_FP64, abi.AP_TIER_DD, abi.AP_TIER_PERTURB}
    assert {m["fractal_type"] for m in META} == {0, 1, 2, 3, 4}
    assert any(m["bbsa_order"] == 8 for m in META)


def test_depth_rule():
    base = 700
    assert engine.get_adaptive_max_iter_from_probe(np.full((4, 4), -1.0, np.float32), base) == base
    it = np.array([[-1.0, 10.0], [20.0, 30.0]], np.float32)
    # max(1.35 * p98, 1.2 * max) with numpy's linear percentile, floored at 100
    assert engine.get_adaptive_max_iter_from_probe(it, base) == 100
    it = np.linspace(0, 1000, 101, dtype=np.float32).reshape(1, -1)
    assert engine.get_adaptive_max_iter_from_probe(it, base) == int(max(980.0 * 1.35, 1000.0 * 1.2))
    assert probe_search(100) == 1000 and probe_search(4000) == 8000


def test_plan_keeps_series_settings_on_the_floatexp_tier():
    """A frame maps FloatExp views to chained BLA (order 32, tol <= 1e-6); the probe keeps
    the caller's series settings and leaps nowhere."""
    from decimal import Decimal
    m = next(x for x in META if x["name"] == "pert_cfg3")
    p, orbit = engine.plan_probe(Decimal(m["cx"]), Decimal(m["cy"]), Decimal("1e-1000"), 2000, 16, 9,
                                 arith="ref_cuda")
    assert p.tier == abi.AP_TIER_FLOATEXP and p.bla_levels == 0 and p.strict_glitch == 0
    assert p.flags == abi.AP_FLAG_NO_RGB | abi.AP_FLAG_ESCAPE_GLITCH
    assert p.e_scale > 0 and p.bbsa_inv_r != 1.0
    assert p.ref_px == pytest.approx(15 * float(0.5), abs=8.0)
    assert orbit[2] > 0
