"""The native decimal arithmetic (ap_decimal_arith, ap_decimal_escape) against
Python's decimal module, which the reference's Decimal orbits use
(math_core/high_precision.py:581-703): every +, - and * exact, then rounded to P
significant digits, half to even.  Random operands, crafted ties and carries, long
and short operands, far-apart exponents, signed zeros; then whole escape loops of
every formula, including bounded chaotic orbits."""
import ctypes as C
import os
from decimal import Decimal, localcontext

import numpy as np
import pytest

from fractura_b200 import _lib
from fractura_b200 import high_precision as hp

pytestmark = pytest.mark.skipif(not os.path.exists(_lib.LIB_PATH), reason="engine library not built")


def _enc(d):
    s, e, limbs = hp._dec_parts(d)
    return np.array([s, e, len(limbs)], np.int64), np.array(limbs, np.uint64)


def _dec(meta, limbs):
    n = int(meta[2])
    coef = "".join(f"{int(x):08d}" for x in limbs[:n][::-1]).lstrip("0") or "0"
    return Decimal((int(meta[0]), tuple(int(c) for c in coef), int(meta[1])))


def native(op, a, b, prec):
    L = _lib.load()
    am, al = _enc(a)
    bm, bl = _enc(b)
    om = np.zeros(3, np.int64)
    ol = np.zeros(400, np.uint64)
    c = C.c_int32(0)
    _lib.check(L.ap_decimal_arith(op, am.ctypes.data_as(C.c_void_p), al.ctypes.data_as(C.c_void_p),
                                  bm.ctypes.data_as(C.c_void_p), bl.ctypes.data_as(C.c_void_p), prec,
                                  om.ctypes.data_as(C.c_void_p), ol.ctypes.data_as(C.c_void_p), C.byref(c)),
               "ap_decimal_arith")
    return c.value if op == 3 else _dec(om, ol)


def python(op, a, b, prec):
    with localcontext() as ctx:
        ctx.prec = prec
        if op == 0:
            return a + b
        if op == 1:
            return a - b
        if op == 2:
            return a * b
        return (a > b) - (a < b)


def same(x, y):
    """Equal values and equal signs (also of zeros)."""
    return x == y and x.is_signed() == y.is_signed()


def _rand_dec(rng, max_digits=120, exp_range=(-200, 20)):
    nd = int(rng.integers(1, max_digits))
    digits = "".join(str(int(d)) for d in rng.integers(0, 10, nd))
    e = int(rng.integers(*exp_range))
    sign = int(rng.integers(0, 2))
    return Decimal((sign, tuple(int(c) for c in digits), e))


@pytest.mark.parametrize("prec", [1, 7, 8, 9, 50, 110, 229])
def test_random_operations_equal_the_decimal_module(prec):
    rng = np.random.default_rng(prec)
    for _ in range(600):
        a, b = _rand_dec(rng), _rand_dec(rng)
        if rng.random() < 0.3:  # nearby magnitudes: cancellation
            b = -a + _rand_dec(rng, 20, (-240, -150))
        for op in (0, 1, 2, 3):
            got, want = native(op, a, b, prec), python(op, a, b, prec)
            if op == 3:
                assert got == want, (a, b)
            else:
                assert same(got, want), (op, a, b, prec, got, want)


@pytest.mark.parametrize("prec", [3, 8, 16, 40])
def test_ties_carries_and_gaps(prec):
    D = Decimal
    cases = []
    base = "9" * prec
    cases += [(D(base), D(1)), (D(base), D("0.5")), (D(base + "5"), D(0)), (D("1" + "0" * prec + "5"), D(0))]
    cases += [(D("2" + "0" * (prec - 1) + "5"), D(0)), (D("3" + "0" * (prec - 1) + "5"), D(0))]  # half-even
    cases += [(D("1" + "0" * (prec - 1) + "5"), D("1e-300")), (D("1" + "0" * (prec - 1) + "5"), D("-1e-300"))]
    cases += [(D("1"), D("-1e-400")), (D("1" + "0" * prec), D("-1e-400")), (D("1e50"), D("-1e-50"))]
    cases += [(D(0), D(0)), (D("-0"), D("-0")), (D("-0"), D(0)), (D("1.5"), D("-1.5")), (D("-0"), D("-3"))]
    cases += [(D("5e-1000"), D("5e-1000")), (D("12345678901234567890123456789"), D("-1e-30"))]
    for a, b in cases:
        for op in (0, 1, 2, 3):
            got, want = native(op, a, b, prec), python(op, a, b, prec)
            if op == 3:
                assert got == want, (a, b)
            else:
                assert same(got, want), (op, a, b, prec, got, want)


FORMULAS = [(0, 0.0, 0.0, 3), (1, 0.0, 0.0, 3), (2, -0.8, 0.156, 3), (3, -1.755, 0.03, 3),
            (4, 0.0, 0.0, 3), (4, 0.0, 0.0, 5)]


@pytest.mark.parametrize("formula", FORMULAS, ids=lambda f: f"type{f[0]}_n{f[3]}")
@pytest.mark.parametrize("prec_bits", [150, 400])
def test_escape_loops_equal_the_python_loop(formula, prec_bits):
    ft, jx, jy, n = formula
    rng = np.random.default_rng(prec_bits + 7 * ft + n)
    for _ in range(8):
        if ft in (2, 3):
            x, y = rng.uniform(-1.5, 1.5), rng.uniform(-1.0, 1.0)
        else:
            x, y = rng.uniform(-2.0, 0.6), rng.uniform(-1.2, 1.2)
        cx = Decimal(repr(x)) + Decimal(int(rng.integers(1, 10 ** 9))).scaleb(-int(rng.integers(20, 90)))
        cy = Decimal(repr(y)) - Decimal(int(rng.integers(1, 10 ** 9))).scaleb(-int(rng.integers(20, 90)))
        got = hp.decimal_escape_scalar(cx, cy, 1500, ft, jx, jy, prec_bits, n, 0.1, 0.2)
        want = hp.decimal_escape_scalar_py(cx, cy, 1500, ft, jx, jy, prec_bits, n, 0.1, 0.2)
        assert got == want, (cx, cy, got, want)


def native_float(d):
    L = _lib.load()
    m, limbs = _enc(d)
    out = C.c_double(0.0)
    rc = L.ap_decimal_to_double(m.ctypes.data_as(C.c_void_p), limbs.ctypes.data_as(C.c_void_p), C.byref(out))
    return None if rc != 0 else out.value


def test_conversion_equals_float_of_decimal():
    """Correctly rounded float64 of decimals of every length and of the scales orbits
    produce (1e-300 .. 1e30); undecided only at ties or within ~2^-110 of one, and
    above 2^127 (values no orbit reaches), where the decimal module converts."""
    rng = np.random.default_rng(11)
    undecided = 0
    for _ in range(20000):
        d = _rand_dec(rng, max_digits=int(rng.integers(2, 700)), exp_range=(-400, 5))
        if not (Decimal("1e-300") < abs(d) < Decimal("1e300")):
            continue
        got = native_float(d)
        if got is None:
            undecided += abs(d) < Decimal("1e30")
            continue
        want = float(d)
        assert got == want and np.signbit(got) == np.signbit(want), (d, got, want)
    assert undecided == 0
    # exact values, ties and their neighbours
    for x in (1.0, 0.1, 1e-80, 3.0e-300, 65536.0, 123456.789, -2.5e-17):
        d = Decimal(x)  # the exact binary value
        assert native_float(d) == x
        nxt = np.nextafter(x, np.inf)
        half = (Decimal(x) + Decimal(float(nxt))) / 2  # an exact tie
        assert native_float(half) in (None, float(half))
        for eps in (Decimal("1e-400"), -Decimal("1e-400")):
            assert native_float(half + eps) in (None, float(half + eps))
    assert native_float(Decimal("-0")) == 0.0 and np.signbit(native_float(Decimal("-0")))


@pytest.mark.parametrize("formula", FORMULAS, ids=lambda f: f"type{f[0]}_n{f[3]}")
@pytest.mark.parametrize("prec_bits", [150, 400])
def test_orbit_loops_equal_the_python_loop(formula, prec_bits):
    ft, jx, jy, n = formula
    rng = np.random.default_rng(3 * prec_bits + 7 * ft + n)
    for _ in range(6):
        if ft in (2, 3):
            x, y = rng.uniform(-1.5, 1.5), rng.uniform(-1.0, 1.0)
        else:
            x, y = rng.uniform(-2.0, 0.6), rng.uniform(-1.2, 1.2)
        cx = Decimal(repr(x)) + Decimal(int(rng.integers(1, 10 ** 9))).scaleb(-int(rng.integers(20, 90)))
        cy = Decimal(repr(y)) - Decimal(int(rng.integers(1, 10 ** 9))).scaleb(-int(rng.integers(20, 90)))
        got = hp.decimal_orbit(cx, cy, 1500, ft, jx, jy, prec_bits, n, 0.1, 0.2)
        want = hp.decimal_orbit_py(cx, cy, 1500, ft, jx, jy, prec_bits, n, 0.1, 0.2)
        assert got[2] == want[2]
        assert np.array_equal(got[0].view(np.uint64), want[0].view(np.uint64))
        assert np.array_equal(got[1].view(np.uint64), want[1].view(np.uint64))


@pytest.mark.parametrize("c", [("0", "0"), ("-1", "0"), ("-0.1", "0.1"), ("-1.3", "0.05"), ("0.25", "0")])
def test_periodic_orbits_equal_the_python_loop(c):
    cx, cy = Decimal(c[0]), Decimal(c[1])
    got = hp.decimal_orbit(cx, cy, 5000, 0, 0.0, 0.0, 300)
    want = hp.decimal_orbit_py(cx, cy, 5000, 0, 0.0, 0.0, 300)
    assert got[2] == want[2] == 5000
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
