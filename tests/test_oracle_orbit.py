"""The oracle's reference-orbit search (oracle/ref_orbit.py) against orbits the reference
itself computed (tests/golden/pert_samples.npz, fexp_samples.npz): the same reference
position (u, v), escape step and float64 orbit, bit for bit."""
from decimal import Decimal, localcontext

import numpy as np
import pytest

import ref_orbit
from helpers import load_golden

PS, PMETA = load_golden("pert_samples.npz")
FS, FMETA = load_golden("fexp_samples.npz")
CASES = [("pert", m["name"]) for m in PMETA] + [("fexp", m["name"]) for m in FMETA if m["name"] != "fexp_cfg3"]


@pytest.mark.parametrize("src,name", CASES)
def test_find_reference_matches_reference_orbits(src, name):
    G, META = (PS, PMETA) if src == "pert" else (FS, FMETA)
    m = next(x for x in META if x["name"] == name)
    pw = Decimal(m["width"])
    with localcontext() as ctx:
        ctx.prec = ref_orbit.view_digits(pw)
        ph = pw * (Decimal(m["H"]) / Decimal(m["W"]))
    cx, cy, u, v, re, im, rl = ref_orbit.find_reference(
        Decimal(m["cx"]), Decimal(m["cy"]), pw, ph, m["max_iter"], ft=m["fractal_type"],
        julia_cx=m["julia_cx"], julia_cy=m["julia_cy"], n=m["gen_n"], kr=m["gen_kr"], ki=m["gen_ki"])
    want_re, want_im = G[name + "__re"], G[name + "__im"]
    assert rl == len(want_re) - 1
    if "u" in m:
        assert (u, v) == (m["u"], m["v"])
    assert np.array_equal(re[:rl + 1].view(np.uint64), want_re.view(np.uint64))
    assert np.array_equal(im[:rl + 1].view(np.uint64), want_im.view(np.uint64))
