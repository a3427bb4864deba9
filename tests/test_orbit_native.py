"""Reference orbits computed natively (ap_reference_orbit at two fixed-point
precisions bracketing the reference's Decimal precision, Decimal only when those
disagree) against the Decimal loop in the reference's operation order.

The reference's own orbits pin the result (tests/test_oracle_pert.py and
tests/test_oracle_fexp.py compare find_optimal_reference_orbit with them).  Here:
seeded points of every formula at two precisions give float64 orbits, escape
steps and escape values equal to the Decimal loop's, including bounded chaotic
orbits that run through the available precision; interior points whose orbits
become exactly periodic reach the same cycle and the same ref_len.
"""
from decimal import Decimal, localcontext

import numpy as np
import pytest

from fractura_b200 import high_precision as hp

FORMULAS = [  # fractal_type, julia, gen_n, kr, ki
    (0, (0.0, 0.0), 3, 0.25, 1.0),
    (1, (0.0, 0.0), 3, 0.25, 1.0),
    (2, (-0.8, 0.156), 3, 0.25, 1.0),
    (3, (-1.755, 0.03), 3, 0.25, 1.0),
    (4, (0.0, 0.0), 3, 0.1, 0.2),
    (4, (0.0, 0.0), 5, 0.1, 0.2),
]


def _points(seed, n, ft):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        if ft in (2, 3):
            x, y = rng.uniform(-1.5, 1.5), rng.uniform(-1.0, 1.0)
        else:
            x, y = rng.uniform(-2.0, 0.6), rng.uniform(-1.2, 1.2)
        digits = int(rng.integers(20, 120))
        out.append((Decimal(repr(x)) + Decimal(int(rng.integers(1, 10 ** 9))).scaleb(-digits),
                    Decimal(repr(y)) - Decimal(int(rng.integers(1, 10 ** 9))).scaleb(-digits)))
    return out


@pytest.mark.parametrize("prec_bits", [256, 700])
@pytest.mark.parametrize("formula", FORMULAS, ids=lambda f: f"type{f[0]}_n{f[2]}")
def test_orbits_equal_decimal(formula, prec_bits):
    ft, (jx, jy), n, kr, ki = formula
    for cx, cy in _points(prec_bits + 31 * ft + n, 6, ft):
        a = hp.compute_single_highprec_orbit(cx, cy, 3000, ft, jx, jy, prec_bits, n, kr, ki)
        b = hp.decimal_orbit(cx, cy, 3000, ft, jx, jy, prec_bits, n, kr, ki)
        assert a[2] == b[2]
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        ea = hp.compute_highprec_escape_scalar(cx, cy, 3000, ft, jx, jy, prec_bits, n, kr, ki)
        eb = hp.decimal_escape_scalar(cx, cy, 3000, ft, jx, jy, prec_bits, n, kr, ki)
        assert ea == eb
        # the probe's single pair of runs gives the same value and, when certified,
        # the same orbit
        ep, orbit = hp.probe_candidate(cx, cy, 3000, ft, jx, jy, prec_bits, n, kr, ki)
        assert ep == eb
        if orbit is not None:
            assert orbit[2] == b[2] and np.array_equal(orbit[0], b[0]) and np.array_equal(orbit[1], b[1])


@pytest.mark.parametrize("c", [("0", "0"), ("-1", "0"), ("0", "1"), ("-0.1", "0.1"),
                               ("-1.3", "0.05"), ("0.25", "0")])
def test_periodic_interior_orbits(c):
    cx, cy = Decimal(c[0]), Decimal(c[1])
    a = hp.compute_single_highprec_orbit(cx, cy, 5000, 0, 0.0, 0.0, 300)
    b = hp.decimal_orbit(cx, cy, 5000, 0, 0.0, 0.0, 300)
    assert a[2] == b[2] == 5000
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_uncertified_orbit_takes_the_decimal_path():
    """A bounded chaotic Burning Ship orbit at 256 bits: the two fixed-point runs part
    after ~900 steps, and the result is the Decimal loop's."""
    from test_orbit_native import _points as pts
    cx, cy = pts(256 + 31, 6, 1)[3]
    lo, hi = hp.orbit_limbs(256)

    def seeds(L, I):
        return hp._seeds(1, cx, cy, 0.0, 0.0, 0.25, 1.0, L, I)

    a = hp._native_orbit(seeds, hi, 3000, 1, 3)
    b = hp._native_orbit(seeds, lo, 3000, 1, 3)
    assert not np.array_equal(a[0], b[0])
    got = hp.compute_single_highprec_orbit(cx, cy, 3000, 1, 0.0, 0.0, 256)
    ref = hp.decimal_orbit(cx, cy, 3000, 1, 0.0, 0.0, 256)
    assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
    esc, orbit = hp.probe_candidate(cx, cy, 3000, 1, 0.0, 0.0, 256)
    assert orbit is None and esc == hp.decimal_escape_scalar(cx, cy, 3000, 1, 0.0, 0.0, 256)


SEARCH_VIEWS = {  # centre kept / a probe candidate wins (its orbit is reused)
    "mandelbrot": ("-0.7436438870371587", "0.1318259042053119", "1e-12", 0, 20000),
    "ship": ("-1.7692733407791943", "0.01796380726768093", "2e-14", 1, 6000),
}


@pytest.mark.parametrize("view", sorted(SEARCH_VIEWS))
@pytest.mark.parametrize("speculate", [False, True])
def test_reference_search_is_the_sequential_one(view, speculate):
    """find_optimal_reference_orbit, with the probe beside the centre orbit or after
    it, picks the reference the sequential Decimal search picks, with its orbit."""
    cxs, cys, ws, ft, mi = SEARCH_VIEWS[view]
    cx, cy, pw = Decimal(cxs), Decimal(cys), Decimal(ws)
    ph = pw * Decimal(9) / Decimal(16)
    hp.clear_reference_orbit_cache()
    got = hp.find_optimal_reference_orbit(cx, cy, pw, ph, mi, 160, 90, fractal_type=ft, speculate=speculate)
    hp.clear_reference_orbit_cache()
    bits = hp.compute_required_prec_bits(pw)
    centre = hp.decimal_orbit(cx, cy, mi, ft, 0.0, 0.0, bits)
    assert centre[2] < int(0.6 * mi)  # the probe decides
    best_esc, best = max(int(centre[2] * 1.2), centre[2] + 32), None
    x_min, y_max = cx - pw / 2, cy + ph / 2
    for u, v in hp.PROBE_UV:
        x, y = x_min + Decimal(str(u)) * pw, y_max - Decimal(str(v)) * ph
        e = hp.decimal_escape_scalar(x, y, mi, ft, 0.0, 0.0, bits)
        if e > best_esc:
            best_esc, best = e, (x, y, u, v)
    want = centre
    if best is not None:
        cand = hp.decimal_orbit(best[0], best[1], mi, ft, 0.0, 0.0, bits)
        if cand[2] > centre[2]:
            want = cand
            assert (got[0], got[1], got[2], got[3]) == best
    assert (best is not None) == (view == "ship")
    assert got[6] == want[2]
    assert np.array_equal(got[4][:want[2] + 1], want[0][:want[2] + 1])
    assert np.array_equal(got[5][:want[2] + 1], want[1][:want[2] + 1])


def test_fixed_point_conversion():
    L = 4
    for v in ("0", "1", "-1", "0.5", "-0.75", "255.125", "-3.14159265358979323846264338327950288"):
        limbs = hp.to_fixed(Decimal(v), L)
        q = int.from_bytes(limbs.tobytes(), "little")
        if q >= 1 << (64 * L - 1):
            q -= 1 << (64 * L)
        with localcontext() as ctx:
            ctx.prec = 200
            assert abs(Decimal(q) / Decimal(2) ** (64 * (L - 1)) - Decimal(v)) <= Decimal(2) ** -(64 * (L - 1))
    with pytest.raises(OverflowError):
        hp.to_fixed(Decimal(2) ** 70, 2)
    assert [hp.orbit_int_limbs(t, n) for t, n in ((0, 3), (1, 3), (4, 3), (4, 4), (4, 8))] == [1, 1, 1, 2, 3]


@pytest.mark.parametrize("int_limbs", [1, 2])
@pytest.mark.parametrize("fractal_type,gen_n", [(0, 2), (1, 2), (4, 5)])
def test_fixed_size_products_at_every_size(fractal_type, gen_n, int_limbs):
    """The products with compile-time limb counts (3-24 limbs) give the orbit the
    runtime-bound products give: a point that escapes within a few dozen steps has the
    same float64 orbit at every precision with 64 or more fractional bits beyond a
    double's, so each table size must match the 40-limb run (runtime path) exactly."""
    need = hp.orbit_int_limbs(fractal_type, gen_n)
    if int_limbs < need:
        pytest.skip("needs more integer limbs")
    # just past the cusp at 1/4 (about 30 steps), and an outer Multibrot point
    cx, cy = Decimal("0.2600000000000000123"), Decimal("0.0010000000000000456")
    if fractal_type == 4:
        cx, cy = Decimal("0.41"), Decimal("0.53")

    import ctypes as C
    from fractura_b200 import _lib
    lib = hp._native()

    def run(L):
        sd = hp._seeds(fractal_type, cx, cy, 0.0, 0.0, 0.25, 1.0, L, int_limbs)
        re, im = np.zeros(401), np.zeros(401)
        n, m2 = C.c_int32(0), C.c_double(0.0)
        _lib.check(lib.ap_reference_orbit(sd.ctypes.data_as(C.c_void_p), L, int_limbs, fractal_type, gen_n, 400,
                                          0, re.ctypes.data_as(C.c_void_p), im.ctypes.data_as(C.c_void_p),
                                          C.byref(n), C.byref(m2), None), "ap_reference_orbit")
        return re, im, n.value

    want = run(40)  # beyond the fixed-size table: the runtime-bound products
    assert 2 < want[2] < 400
    k = want[2] + 1
    for L in range(int_limbs + 2, 25):
        re, im, n = run(L)
        assert n == want[2], (L, n, want[2])
        assert np.array_equal(re[:k], want[0][:k]) and np.array_equal(im[:k], want[1][:k]), L


@pytest.mark.parametrize("prec_bits", [256, 700])
@pytest.mark.parametrize("formula", FORMULAS, ids=lambda f: f"type{f[0]}_n{f[2]}")
def test_certified_runs_equal_decimal(formula, prec_bits):
    """ap_reference_orbit_cert: wherever its error bound certifies a run (64 fractional
    bits below or above the Decimal precision), the float64 orbit, the escape step and
    |Z|^2 at escape equal the Decimal loop's; and most seeded runs (non-chaotic orbits)
    are certified, so the search needs one run per orbit."""
    ft, (jx, jy), n, kr, ki = formula
    lo, hi = hp.orbit_limbs(prec_bits, hp.orbit_int_limbs(ft, n))
    certified = 0
    pts = _points(prec_bits + 7 * ft + n, 8, ft)
    for cx, cy in pts:
        seeds = hp._Seeds(ft, cx, cy, jx, jy, kr, ki)
        b = None
        for L in (lo, hi):  # below and above the Decimal precision
            a = hp._first_run(seeds, L, 3000, ft, n, prec_bits)
            if not a[4]:
                continue
            certified += 1
            if b is None:
                b = hp.decimal_orbit_py(cx, cy, 3000, ft, jx, jy, prec_bits, n, kr, ki)
            assert a[2] == b[2] and np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
            if a[2] < 3000:
                assert hp._smooth_escape(a[2], a[3], 3000, ft, n) == hp.decimal_escape_scalar(
                    cx, cy, 3000, ft, jx, jy, prec_bits, n, kr, ki)
    assert certified >= len(pts), certified


def test_certification_refuses_a_run_that_differs_from_decimal():
    """The centre of the Burning Ship golden view at 2e-14: its fixed-point run leaves the
    Decimal orbit before the escape, and the bound does not certify it."""
    cx, cy, bits = Decimal("-1.7692733407791943"), Decimal("0.01796380726768093"), 174
    lo, hi = hp.orbit_limbs(bits, hp.orbit_int_limbs(1, 3))
    b = hp.decimal_orbit_py(cx, cy, 6000, 1, 0.0, 0.0, bits)
    for L in (lo, hi):
        a = hp._first_run(hp._Seeds(1, cx, cy, 0.0, 0.0, 0.25, 1.0), L, 6000, 1, 3, bits)
        assert not (a[2] == b[2] and np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]))
        assert not a[4]
    got = hp.compute_single_highprec_orbit(cx, cy, 6000, 1, 0.0, 0.0, bits)
    assert got[2] == b[2] and np.array_equal(got[0], b[0]) and np.array_equal(got[1], b[1])
