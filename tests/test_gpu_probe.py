"""Adaptive max-iter probe on the device (engine.probe_iter_map / probe_adaptive_max_iter).

* CPU profile: the device's probe map equals the reference's CPU probe map value for
  value on every fixture (FP64, DD and perturbation views of all five formulas), and
  the depth equals the one the reference returned.
* CUDA profile: device == oracle on the same planned pass.
* FloatExp views (no reference CPU fixture: that branch of the reference fails to
  compile in Numba): device == oracle in both profiles.
"""
from decimal import Decimal

import numpy as np
import pytest

from fractura_b200 import abi, engine
from fractura_b200 import high_precision as hp
from helpers import load_golden, oracle_probe, probe_args

pytestmark = pytest.mark.gpu

G, META = load_golden("probe.npz")


def device_probe(m, arith):
    hp.clear_reference_orbit_cache()
    return engine.probe_iter_map(*probe_args(m), arith=arith)


@pytest.mark.parametrize("name", [m["name"] for m in META])
def test_probe_map_device_equals_reference(name):
    m = next(x for x in META if x["name"] == name)
    it = device_probe(m, "ref_cpu")
    want = G[name + "__iter"]
    assert np.array_equal(it.view(np.uint32), want.view(np.uint32)), \
        int((it.view(np.uint32) != want.view(np.uint32)).sum())
    hp.clear_reference_orbit_cache()
    depth = engine.probe_adaptive_max_iter(
        Decimal(m["cx"]), Decimal(m["cy"]), Decimal(m["width"]), m["base_iter"], target_w=m["W"],
        target_h=m["H"], fractal_type=m["fractal_type"], julia_cx=m["julia_cx"], julia_cy=m["julia_cy"],
        gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"], precision_mode=m["precision_mode"],
        bbsa_tol=m["bbsa_tol"], bbsa_order=m["bbsa_order"])
    assert depth == m["depth"]


@pytest.mark.parametrize("name", [m["name"] for m in META])
def test_probe_map_device_equals_oracle_cuda_profile(name):
    m = next(x for x in META if x["name"] == name)
    it = device_probe(m, "ref_cuda")
    want = oracle_probe(m, abi.AP_ARITH_REF_CUDA)
    assert np.array_equal(it.view(np.uint32), want.view(np.uint32)), \
        int((it.view(np.uint32) != want.view(np.uint32)).sum())


@pytest.mark.parametrize("arith", ["ref_cpu", "ref_cuda"])
def test_floatexp_probe_device_equals_oracle(arith):
    base = next(x for x in META if x["name"] == "pert_cfg3")
    m = dict(base, width="1e-1000", W=32, H=18, base_iter=5000, name="fexp_cfg3")
    assert engine.select_tier(Decimal(m["width"]), m["precision_mode"]) == abi.AP_TIER_FLOATEXP
    it = device_probe(m, arith)
    want = oracle_probe(m, abi.AP_ARITH_REF_CPU if arith == "ref_cpu" else abi.AP_ARITH_REF_CUDA)
    assert np.array_equal(it.view(np.uint32), want.view(np.uint32))
    assert (it >= 0).any()


def test_dynamic_max_iter_adaptive_mode_runs_the_probe():
    m = next(x for x in META if x["name"] == "pert_julia")
    hp.clear_reference_orbit_cache()
    got = engine.compute_dynamic_max_iter(
        m["base_iter"], Decimal(m["width"]), "Adaptive (Probe)", Decimal(m["cx"]), Decimal(m["cy"]),
        target_w=m["W"], target_h=m["H"], fractal_type=m["fractal_type"], julia_cx=m["julia_cx"],
        julia_cy=m["julia_cy"], gen_n=m["gen_n"], gen_kr=m["gen_kr"], gen_ki=m["gen_ki"],
        precision_mode=m["precision_mode"], bbsa_tol=m["bbsa_tol"], bbsa_order=m["bbsa_order"])
    assert got == m["depth"]
