"""The dc-aware chained-BLA table (oracle apo_build_bla_dc, the engine's bla_form="accurate").

Checked on the config-3 reference orbit of the goldens (1e-160 view, 8050 steps):
  * with dc_max = 0 the table is the reference's level 0 and a merge that only
    differs from the reference's by its radius rule;
  * radii never increase with the level;
  * every leap taken from inside its radius, with |dc| up to dc_max, agrees with
    stepping the same iterations one by one (FP64 perturbation steps) to 1e-12
    relative: the leap's dropped quadratic terms stay at the per-step tolerance.
"""
import numpy as np

import oracle
from fractura_b200.config import ACCURATE_BLA_EPS
from helpers import load_golden

G, META = load_golden("pert_samples.npz")
M = next(m for m in META if m["name"] == "cfg3")
RE, IM, RL = G["cfg3__re"], G["cfg3__im"], M["ref_len"]
DC_MAX = 0.6 * float(M["width"])  # beyond the frame's largest |dc|


def _table(dc_max):
    return oracle.build_bla_dc(RE, IM, RL, 0, ACCURATE_BLA_EPS, dc_max, 16, 3, 0.25, 1.0)


def test_level0_is_the_reference_level0():
    T = _table(0.0)
    R = oracle.build_bla(RE, IM, RL, 0, ACCURATE_BLA_EPS, 16, 3, 0.25, 1.0)
    assert T[0].tobytes() == R[0].tobytes()
    # coefficients of every entry both tables keep are the same products
    both = (T[:, :, 4] > 0) & (R[:, :, 4] > 0)
    assert np.array_equal(T[both][:, :4], R[both][:, :4])


def test_radii_non_increasing_with_level():
    T = _table(DC_MAX)
    assert np.all(np.diff(T[:, :, 4], axis=0) <= 0)
    assert np.count_nonzero(T[11, :, 4]) > 0  # leaps of 2^11 steps remain valid


def test_leaps_agree_with_single_steps():
    T = _table(DC_MAX)
    Z = RE + 1j * IM
    rng = np.random.default_rng(20261203)
    worst = 0.0
    n = 0
    for d in range(1, 16):
        ks = np.flatnonzero(T[d, :, 4] > 0)
        if ks.size == 0:
            continue
        for k in rng.choice(ks, size=min(4, ks.size), replace=False):
            r = np.sqrt(T[d, k, 4])
            dz = 0.999 * r * np.exp(2j * np.pi * rng.random())
            dc = DC_MAX * rng.random() * np.exp(2j * np.pi * rng.random())
            A = T[d, k, 0] + 1j * T[d, k, 1]
            B = T[d, k, 2] + 1j * T[d, k, 3]
            leap = A * dz + B * dc
            x = dz
            for t in range(k, k + (1 << d)):
                x = 2.0 * Z[t] * x + x * x + dc
            worst = max(worst, abs(leap - x) / abs(x))
            n += 1
    assert n > 20
    assert worst <= 1e-12, worst
