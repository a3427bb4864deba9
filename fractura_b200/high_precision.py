"""Host-side high-precision inputs of the perturbation tiers.

Restates math_core/high_precision.py's reference-orbit machinery.  The
reference iterates orbits in Decimal (its path when gmpy2 is absent,
math_core/high_precision.py:657-703 and :802-873); here the orbit loop runs in
native binary fixed point with more bits than those Decimal digits
(ap_reference_orbit, host code of the library), and the orbit arrays equal the
reference's:

  compute_single_highprec_orbit   math_core/high_precision.py:706-875
  compute_highprec_escape_scalar  math_core/high_precision.py:581-703
  find_optimal_reference_orbit    math_core/high_precision.py:919-1097
  cache_reference_orbit / clear_reference_orbit_cache (16-entry LRU)

Every Decimal computation runs in a local context; the caller's context is
never modified.
"""
import math
import os
import threading
from concurrent.futures import ThreadPoolExecutor
from decimal import Decimal, localcontext

import numpy as np

from .config import INV_LN2_F32, LN_BAILOUT_LOG, compute_required_prec_bits, decimal_context

_ORBIT_CACHE = []
_ORBIT_LOCK = threading.Lock()
_CACHE_SIZE = 16


def _orbit_digits(prec_bits):
    """Decimal digits the reference's orbit uses (math_core/high_precision.py:720)."""
    return int(prec_bits / 3.32) + 30


def orbit_int_limbs(fractal_type, gen_n):
    """Integer limbs of the fixed-point orbit: room for |Z|^2 of the first escaped Z
    (|Z| <= 256 the step before, so at most about 2^(16 n) for z^n), plus the sign."""
    n = max(int(gen_n), 2) if fractal_type == 4 else 2
    return (16 * n + 8 + 1 + 63) // 64


def orbit_limbs(prec_bits, int_limbs=1):
    """(low, high) limb counts of the two fixed-point orbits: 64 fractional bits fewer
    and at least 64 more than the reference's Decimal precision, plus int_limbs."""
    dec_bits = _orbit_digits(prec_bits) * 3.3219280948873626
    lo = max(1, int(math.floor((dec_bits - 64.0) / 64.0)))
    hi = int(math.ceil((dec_bits + 64.0) / 64.0))
    return lo + int_limbs, hi + int_limbs


def _ratio(value):
    """A Decimal (or a number's str) as the exact fraction (num, den), den > 0."""
    d = value if isinstance(value, Decimal) else Decimal(str(value))
    return d.as_integer_ratio()


def _fixed_from_ratio(num, den, limbs, int_limbs=1):
    shift = 64 * (limbs - int_limbs)
    q, r = divmod(abs(num) << shift, den)
    if 2 * r > den or (2 * r == den and q & 1):
        q += 1
    if num < 0:
        q = -q
    if not -(1 << (64 * limbs - 1)) <= q < (1 << (64 * limbs - 1)):
        raise OverflowError("value outside the fixed-point range")
    return np.frombuffer((q % (1 << (64 * limbs))).to_bytes(8 * limbs, "little"), dtype=np.uint64)


def to_fixed(value, limbs, int_limbs=1):
    """A Decimal (or a number's str) as two's-complement fixed point,
    value * 2^(64 (limbs - int_limbs)) rounded half to even, in little-endian uint64 limbs."""
    return _fixed_from_ratio(*_ratio(value), limbs, int_limbs)


def _seed_values(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy, gen_kr, gen_ki):
    """(z0, c, K) of the orbit, as the reference starts it (math_core/high_precision.py:722-735)."""
    if fractal_type in (2, 3):
        z0x, z0y, c_x, c_y = Decimal(cand_cx), Decimal(cand_cy), Decimal(str(julia_cx)), Decimal(str(julia_cy))
    else:
        z0x, z0y, c_x, c_y = Decimal(0), Decimal(0), Decimal(cand_cx), Decimal(cand_cy)
    return (z0x, z0y, c_x, c_y, Decimal(str(gen_kr)), Decimal(str(gen_ki)))


def _seeds(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy, gen_kr, gen_ki, limbs, int_limbs=1):
    """The seeds of one orbit in fixed point with `limbs` limbs."""
    vals = _seed_values(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy, gen_kr, gen_ki)
    return np.ascontiguousarray(np.concatenate([to_fixed(v, limbs, int_limbs) for v in vals]))


class _Seeds:
    """The seeds of one orbit at any limb count: the exact fractions are formed once
    (on first use, by whichever thread gets there first), then rounded per limb count."""

    def __init__(self, fractal_type, cand_cx, cand_cy, julia_cx, julia_cy, gen_kr, gen_ki):
        self.args = (fractal_type, cand_cx, cand_cy, julia_cx, julia_cy, gen_kr, gen_ki)
        self.ratios = None
        self.lock = threading.Lock()

    def __call__(self, limbs, int_limbs=1):
        with self.lock:
            if self.ratios is None:
                self.ratios = [_ratio(v) for v in _seed_values(*self.args)]
        return np.ascontiguousarray(np.concatenate([_fixed_from_ratio(n, d, limbs, int_limbs)
                                                    for n, d in self.ratios]))


def _native():
    from . import _lib
    return _lib.load()


_PROBE_POOL = None
_PAIR_LOCK = threading.Lock()


def _probe_pool():
    """Threads for the centre orbit and the probe candidates of
    find_optimal_reference_orbit (one task per orbit; the native runs release the
    GIL).  At least one thread per orbit of a search (17): with fewer, the last orbit
    waits for a whole run instead of sharing the cores."""
    global _PROBE_POOL
    with _PAIR_LOCK:
        if _PROBE_POOL is None:
            _PROBE_POOL = ThreadPoolExecutor(max_workers=max(1 + len(PROBE_UV), os.cpu_count() or 4),
                                             thread_name_prefix="probe")
        return _PROBE_POOL


def _native_orbit(seeds_fn, L, max_iter, fractal_type, gen_n, with_mag2=False):
    import ctypes as C
    from . import _lib
    I = orbit_int_limbs(fractal_type, gen_n)
    seeds = seeds_fn(L, I)
    ref_re = np.zeros(max_iter + 1, dtype=np.float64)
    ref_im = np.zeros(max_iter + 1, dtype=np.float64)
    ref_len = C.c_int32(0)
    mag2 = C.c_double(0.0)
    _lib.check(_native().ap_reference_orbit(
        seeds.ctypes.data_as(C.c_void_p), L, I, int(fractal_type), int(gen_n), int(max_iter), 0,
        ref_re.ctypes.data_as(C.c_void_p), ref_im.ctypes.data_as(C.c_void_p), C.byref(ref_len),
        C.byref(mag2), None), "ap_reference_orbit")
    if with_mag2:
        return ref_re, ref_im, int(ref_len.value), float(mag2.value)
    return ref_re, ref_im, int(ref_len.value)


def _native_orbit_cert(seeds_fn, L, max_iter, fractal_type, gen_n, dec_digits):
    """The orbit at L limbs with its proof against the Decimal iteration of dec_digits
    digits (ap_reference_orbit_cert): (ref_re, ref_im, ref_len, |Z|^2 at escape, certified)."""
    import ctypes as C
    from . import _lib
    I = orbit_int_limbs(fractal_type, gen_n)
    seeds = seeds_fn(L, I)
    ref_re = np.zeros(max_iter + 1, dtype=np.float64)
    ref_im = np.zeros(max_iter + 1, dtype=np.float64)
    ref_len = C.c_int32(0)
    mag2 = C.c_double(0.0)
    cert = C.c_int32(0)
    _lib.check(_native().ap_reference_orbit_cert(
        seeds.ctypes.data_as(C.c_void_p), L, I, int(fractal_type), int(gen_n), int(max_iter), int(dec_digits),
        ref_re.ctypes.data_as(C.c_void_p), ref_im.ctypes.data_as(C.c_void_p), C.byref(ref_len),
        C.byref(mag2), C.byref(cert)), "ap_reference_orbit_cert")
    return ref_re, ref_im, int(ref_len.value), float(mag2.value), bool(cert.value)


def _first_run(seeds, L, max_iter, fractal_type, gen_n, prec_bits):
    """A run at L limbs with its certificate against the Decimal iteration:
    (ref_re, ref_im, ref_len, |Z|^2 at escape, certified)."""
    return _native_orbit_cert(seeds, L, max_iter, fractal_type, gen_n, _orbit_digits(prec_bits))


def _run_sequence(seeds, lo, hi, max_iter, fractal_type, gen_n, prec_bits):
    """Certified runs from the cheaper up: the lower precision, then the higher one.
    Returns (run, None) for the first certified run, or (higher run, lower run) for the
    two-run comparison when no bound certifies.  The bound counts each run's own
    truncations and the rounding of its seeds, so the cheaper run certifies whenever its
    bits suffice.  (Fewer bits than that do not: the view's depth, which sets the
    Decimal precision, is also what the probe candidates' orbits resolve.)"""
    a = _first_run(seeds, lo, max_iter, fractal_type, gen_n, prec_bits)
    if a[4]:
        return a, None
    b = _first_run(seeds, hi, max_iter, fractal_type, gen_n, prec_bits)
    return (b, None) if b[4] else (b, a)


def compute_single_highprec_orbit(cand_cx_dec, cand_cy_dec, max_iter, fractal_type=0,
                                  julia_cx=0.0, julia_cy=0.0, prec_bits=256,
                                  gen_n=3, gen_kr=0.25, gen_ki=1.0):
    """Reference orbit Z_0..Z_ref_len as float64 arrays of length max_iter + 1.

    ref_len is the step at which |Z|^2 > 65536 (max_iter if it never does).  For
    Mandelbrot and its Julia set an exactly repeating orbit is detected at
    power-of-two checkpoints and its cycle is copied to the end of the arrays
    (math_core/high_precision.py:706-875).

    The orbit runs natively in binary fixed point, first with 64 fractional bits fewer
    than the reference's Decimal digits carry, then, if needed, with 64 more.  Each run
    carries a bound on its distance from the Decimal iteration
    (ap_reference_orbit_cert); where the bound proves every float64 value and bailout
    decision equal, that orbit is returned.  When neither run is certified, they are
    compared: when both give the same float64 orbit, the Decimal orbit, whose
    precision lies between them, gives it too.  When they differ, the orbit has run
    through the available precision (a bounded chaotic orbit): it is then iterated in
    Decimal exactly as the reference does.
    """
    lo, hi = orbit_limbs(prec_bits, orbit_int_limbs(fractal_type, gen_n))
    seeds = _Seeds(fractal_type, cand_cx_dec, cand_cy_dec, julia_cx, julia_cy, gen_kr, gen_ki)
    a, b = _run_sequence(seeds, lo, hi, max_iter, fractal_type, gen_n, prec_bits)
    return _certified_orbit(a, b, cand_cx_dec, cand_cy_dec, max_iter, fractal_type, julia_cx, julia_cy,
                            prec_bits, gen_n, gen_kr, gen_ki)


def _certified_orbit(a, b, cand_cx_dec, cand_cy_dec, max_iter, fractal_type, julia_cx, julia_cy, prec_bits,
                     gen_n, gen_kr, gen_ki):
    """The orbit of the higher-precision run a when it is certified on its own (b None) or
    the lower one b gives the same float64 orbit, else the exact Decimal orbit."""
    if b is None:
        return a[:3]
    n = a[2] + 1  # past ref_len both hold zeros, or the same copied cycle
    if a[2] == b[2] and np.array_equal(a[0][:n], b[0][:n]) and np.array_equal(a[1][:n], b[1][:n]):
        return a[:3]
    return decimal_orbit(cand_cx_dec, cand_cy_dec, max_iter, fractal_type, julia_cx, julia_cy,
                         prec_bits, gen_n, gen_kr, gen_ki)


def _native_escape(seeds_fn, L, max_iter, fractal_type, gen_n):
    import ctypes as C
    from . import _lib
    I = orbit_int_limbs(fractal_type, gen_n)
    seeds = seeds_fn(L, I)
    k = C.c_int32(0)
    mag2 = C.c_double(0.0)
    trace = C.c_uint64(0)
    _lib.check(_native().ap_reference_orbit(
        seeds.ctypes.data_as(C.c_void_p), L, I, int(fractal_type), int(gen_n), int(max_iter), 1,
        None, None, C.byref(k), C.byref(mag2), C.byref(trace)), "ap_reference_orbit")
    return int(k.value), float(mag2.value), int(trace.value)


def compute_highprec_escape_scalar(cand_cx, cand_cy, max_iter, fractal_type=0,
                                   julia_cx=0.0, julia_cy=0.0, prec_bits=256,
                                   gen_n=3, gen_kr=0.25, gen_ki=1.0):
    """Smooth escape value of one point (max_iter if it stays bounded), as
    math_core/high_precision.py:581-703 computes it.  The orbit runs natively at
    two precisions bracketing the reference's (see compute_single_highprec_orbit);
    if they disagree on the float64 trajectory, the escape step or |Z|^2 there, it
    runs in Decimal."""
    lo, hi = orbit_limbs(prec_bits, orbit_int_limbs(fractal_type, gen_n))

    def seeds(L, I):
        return _seeds(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy, gen_kr, gen_ki, L, I)

    a = _native_escape(seeds, hi, max_iter, fractal_type, gen_n)
    if a != _native_escape(seeds, lo, max_iter, fractal_type, gen_n):
        return decimal_escape_scalar(cand_cx, cand_cy, max_iter, fractal_type, julia_cx, julia_cy,
                                     prec_bits, gen_n, gen_kr, gen_ki)
    k, mag2, _ = a
    return _smooth_escape(k, mag2, max_iter, fractal_type, gen_n)


def _smooth_escape(k, mag2, max_iter, fractal_type, gen_n):
    """The escape scalar of math_core/high_precision.py:581-703 from the escape step
    and |Z|^2 there (max_iter when the orbit stays bounded)."""
    if k >= max_iter:
        return float(max_iter)
    inv_n = (1.0 / math.log(float(gen_n))) if (fractal_type == 4 and gen_n > 1) else float(INV_LN2_F32)
    log_mag = math.log(mag2)
    if log_mag > 1.0:
        return float(k + 1.0) - (math.log(0.5 * log_mag) - LN_BAILOUT_LOG) * inv_n
    return float(k)


def probe_candidate(cand_cx, cand_cy, max_iter, fractal_type=0, julia_cx=0.0, julia_cy=0.0,
                    prec_bits=256, gen_n=3, gen_kr=0.25, gen_ki=1.0):
    """(escape scalar, orbit) of one probe candidate: the value
    compute_highprec_escape_scalar returns and the orbit compute_single_highprec_orbit
    returns, from one pair of certified native runs (orbit None when the runs
    disagree; the escape scalar is then the exact Decimal one)."""
    lo, hi = orbit_limbs(prec_bits, orbit_int_limbs(fractal_type, gen_n))
    seeds = _Seeds(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy, gen_kr, gen_ki)
    a, b = _run_sequence(seeds, lo, hi, max_iter, fractal_type, gen_n, prec_bits)
    return _certified_probe(a, b, cand_cx, cand_cy, max_iter, fractal_type, julia_cx, julia_cy, prec_bits,
                            gen_n, gen_kr, gen_ki)


def _certified_probe(a, b, cand_cx, cand_cy, max_iter, fractal_type, julia_cx, julia_cy, prec_bits, gen_n,
                     gen_kr, gen_ki):
    """(escape scalar, orbit) from the higher-precision run a when it is certified on its
    own (b None) or agrees with the lower one b on the float64 orbit and |Z|^2 at escape,
    else (the exact Decimal scalar, None)."""
    if b is None:
        return _smooth_escape(a[2], a[3], max_iter, fractal_type, gen_n), a[:3]
    n = a[2] + 1
    if (a[2] == b[2] and (a[2] >= max_iter or a[3] == b[3]) and np.array_equal(a[0][:n], b[0][:n])
            and np.array_equal(a[1][:n], b[1][:n])):
        return _smooth_escape(a[2], a[3], max_iter, fractal_type, gen_n), a[:3]
    return decimal_escape_scalar(cand_cx, cand_cy, max_iter, fractal_type, julia_cx, julia_cy, prec_bits,
                                 gen_n, gen_kr, gen_ki), None


class _Runs:
    """The certified runs of one orbit (_run_sequence) as one task of a pool."""

    def __init__(self, pool, cand_cx, cand_cy, max_iter, fractal_type, julia_cx, julia_cy, prec_bits, gen_n,
                 gen_kr, gen_ki):
        lo, hi = orbit_limbs(prec_bits, orbit_int_limbs(fractal_type, gen_n))
        seeds = _Seeds(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy, gen_kr, gen_ki)
        self.task = pool.submit(_run_sequence, seeds, lo, hi, max_iter, fractal_type, gen_n, prec_bits)

    def result(self):
        """(certified run, None), or (higher run, lower run) when neither is certified."""
        return self.task.result()

    def cancel(self):
        self.task.cancel()


# Exact Decimal iteration in the reference's operation order: the path for orbits the
# fixed-point runs cannot certify.
def _orbit_context(prec_bits):
    ctx = decimal_context()
    ctx.prec = int(prec_bits / 3.32) + 30
    return ctx


def _start(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy):
    if fractal_type in (2, 3):
        return (Decimal(cand_cx), Decimal(cand_cy), Decimal(str(julia_cx)), Decimal(str(julia_cy)))
    return Decimal(0), Decimal(0), Decimal(cand_cx), Decimal(cand_cy)


def _step(fractal_type, zx, zy, zx2, zy2, c_x, c_y, two, n, kr, ki):
    """One Decimal iteration, in the reference's operation order."""
    if fractal_type in (0, 2):
        return zx2 - zy2 + c_x, two * zx * zy + c_y
    if fractal_type in (1, 3):
        return zx2 - zy2 + c_x, two * abs(zx) * abs(zy) - c_y
    zn_r, zn_i = zx, zy
    for _ in range(n - 1):
        zn_r, zn_i = zn_r * zx - zn_i * zy, zn_r * zy + zn_i * zx
    kz_r = kr * zx - ki * zy
    kz_i = kr * zy + ki * zx
    return zn_r + kz_r + c_x, zn_i + kz_i + c_y


def decimal_orbit(cand_cx_dec, cand_cy_dec, max_iter, fractal_type=0,
                                  julia_cx=0.0, julia_cy=0.0, prec_bits=256,
                                  gen_n=3, gen_kr=0.25, gen_ki=1.0):
    """Reference orbit Z_0..Z_ref_len as float64 arrays of length max_iter + 1.

    ref_len is the step at which |Z|^2 > 65536 in Decimal arithmetic (max_iter
    if it never does).  For Mandelbrot and its Julia set an exactly repeating
    orbit is detected at power-of-two checkpoints and its cycle is copied to
    the end of the arrays.
    """
    import ctypes as C
    ref_re = np.zeros(max_iter + 1, dtype=np.float64)
    ref_im = np.zeros(max_iter + 1, dtype=np.float64)
    # natively (ap_decimal_orbit: the decimal module's arithmetic without the Python
    # lock), unless an operand is longer than it holds or a conversion is undecided
    args = _native_seeds(fractal_type, cand_cx_dec, cand_cy_dec, julia_cx, julia_cy, gen_kr, gen_ki)
    if args is not None:
        meta, limbs, stride = args
        n = C.c_int32(0)
        rc = _native().ap_decimal_orbit(
            meta.ctypes.data_as(C.c_void_p), limbs.ctypes.data_as(C.c_void_p), int(stride),
            int(_orbit_context(prec_bits).prec), int(fractal_type), int(gen_n), int(max_iter),
            ref_re.ctypes.data_as(C.c_void_p), ref_im.ctypes.data_as(C.c_void_p), C.byref(n))
        if rc == 0:
            return ref_re, ref_im, int(n.value)
        ref_re[:] = 0.0
        ref_im[:] = 0.0
    return decimal_orbit_py(cand_cx_dec, cand_cy_dec, max_iter, fractal_type, julia_cx, julia_cy, prec_bits,
                            gen_n, gen_kr, gen_ki)


def decimal_orbit_py(cand_cx_dec, cand_cy_dec, max_iter, fractal_type=0, julia_cx=0.0, julia_cy=0.0,
                     prec_bits=256, gen_n=3, gen_kr=0.25, gen_ki=1.0):
    """The same loop in Python's decimal module (operands of any length)."""
    ref_re = np.zeros(max_iter + 1, dtype=np.float64)
    ref_im = np.zeros(max_iter + 1, dtype=np.float64)
    with localcontext(_orbit_context(prec_bits)):
        bailout = Decimal(65536)
        two = Decimal(2)
        zx, zy, c_x, c_y = _start(fractal_type, cand_cx_dec, cand_cy_dec, julia_cx, julia_cy)
        kr, ki = Decimal(str(gen_kr)), Decimal(str(gen_ki))
        ref_len = max_iter
        periodic = fractal_type in (0, 2)
        check_step, saved_k = 8, 0
        saved_x, saved_y = zx, zy
        for k in range(max_iter):
            ref_re[k], ref_im[k] = float(zx), float(zy)
            zx2, zy2 = zx * zx, zy * zy
            if (zx2 + zy2) > bailout:
                ref_len = k
                break
            if periodic:
                if k == check_step:
                    check_step <<= 1
                    saved_k = k
                    saved_x, saved_y = zx, zy
                elif k > saved_k and zx == saved_x and zy == saved_y:
                    period = k - saved_k
                    if period > 0:
                        for j in range(k, max_iter + 1):
                            ref_re[j] = ref_re[j - period]
                            ref_im[j] = ref_im[j - period]
                        return ref_re, ref_im, max_iter
            zx, zy = _step(fractal_type, zx, zy, zx2, zy2, c_x, c_y, two, gen_n, kr, ki)
        ref_re[ref_len], ref_im[ref_len] = float(zx), float(zy)
    return ref_re, ref_im, ref_len


def _dec_parts(d):
    """(sign, exponent, base-1e8 limbs, little-endian) of a finite Decimal."""
    t = d.as_tuple()
    digits = "".join(map(str, t.digits)) or "0"
    return t.sign, int(t.exponent), [int(digits[max(0, i - 8):i]) for i in range(len(digits), 0, -8)]


def _native_seeds(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy, gen_kr, gen_ki):
    """(meta, limbs, stride) of the six seeds of the native Decimal loops, as _start and
    the reference form them, or None when an operand is longer than they hold."""
    zx, zy, c_x, c_y = _start(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy)
    parts = [_dec_parts(v) for v in (zx, zy, c_x, c_y, Decimal(str(gen_kr)), Decimal(str(gen_ki)))]
    stride = max(len(p[2]) for p in parts)
    if stride > 200:
        return None
    meta = np.array([[p[0], p[1], len(p[2])] for p in parts], dtype=np.int64)
    limbs = np.zeros((6, stride), dtype=np.uint64)
    for q, p in enumerate(parts):
        limbs[q, :len(p[2])] = p[2]
    return meta, limbs, stride


def decimal_escape_scalar(cand_cx, cand_cy, max_iter, fractal_type=0,
                          julia_cx=0.0, julia_cy=0.0, prec_bits=256,
                          gen_n=3, gen_kr=0.25, gen_ki=1.0):
    """Smooth escape value of one point in Decimal arithmetic (max_iter if it stays
    bounded): the loop of math_core/high_precision.py:581-703, run natively
    (ap_decimal_escape, the decimal module's arithmetic without the Python lock) and
    in Python only for operands longer than the native code holds."""
    import ctypes as C
    from . import _lib
    ctx = _orbit_context(prec_bits)
    args = _native_seeds(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy, gen_kr, gen_ki)
    if args is not None:
        meta, limbs, stride = args
        k = C.c_int32(0)
        mag_meta = np.zeros(3, dtype=np.int64)
        mag_limbs = np.zeros(400, dtype=np.uint64)
        rc = _native().ap_decimal_escape(
            meta.ctypes.data_as(C.c_void_p), limbs.ctypes.data_as(C.c_void_p), int(stride), int(ctx.prec),
            int(fractal_type), int(gen_n), int(max_iter), C.byref(k), mag_meta.ctypes.data_as(C.c_void_p),
            mag_limbs.ctypes.data_as(C.c_void_p))
        if rc == 0:
            if k.value >= max_iter:
                return float(max_iter)
            n = int(mag_meta[2])
            coef = "".join(f"{int(x):08d}" for x in mag_limbs[:n][::-1]).lstrip("0") or "0"
            mag2 = Decimal((int(mag_meta[0]), tuple(int(ch) for ch in coef), int(mag_meta[1])))
            inv_n = (1.0 / math.log(float(gen_n))) if (fractal_type == 4 and gen_n > 1) else float(INV_LN2_F32)
            log_mag = math.log(float(mag2))
            if log_mag > 1.0:
                return float(k.value + 1.0) - (math.log(0.5 * log_mag) - LN_BAILOUT_LOG) * inv_n
            return float(k.value)
        _lib.last_error()  # clear: the Python loop below serves the call
    return decimal_escape_scalar_py(cand_cx, cand_cy, max_iter, fractal_type, julia_cx, julia_cy, prec_bits,
                                    gen_n, gen_kr, gen_ki)


def decimal_escape_scalar_py(cand_cx, cand_cy, max_iter, fractal_type=0,
                             julia_cx=0.0, julia_cy=0.0, prec_bits=256,
                             gen_n=3, gen_kr=0.25, gen_ki=1.0):
    """The same loop in Python's decimal module (operands of any length)."""
    with localcontext(_orbit_context(prec_bits)):
        bailout = Decimal(65536)
        two = Decimal(2)
        zx, zy, c_x, c_y = _start(fractal_type, cand_cx, cand_cy, julia_cx, julia_cy)
        kr, ki = Decimal(str(gen_kr)), Decimal(str(gen_ki))
        inv_n = (1.0 / math.log(float(gen_n))) if (fractal_type == 4 and gen_n > 1) else float(INV_LN2_F32)
        for k in range(max_iter):
            zx2, zy2 = zx * zx, zy * zy
            mag2_dec = zx2 + zy2
            if mag2_dec > bailout:
                log_mag = math.log(float(mag2_dec))
                if log_mag > 1.0:
                    return float(k + 1.0) - (math.log(0.5 * log_mag) - LN_BAILOUT_LOG) * inv_n
                return float(k)
            zx, zy = _step(fractal_type, zx, zy, zx2, zy2, c_x, c_y, two, gen_n, kr, ki)
        return float(max_iter)


def clear_reference_orbit_cache():
    """Drop every cached reference orbit."""
    with _ORBIT_LOCK:
        _ORBIT_CACHE.clear()


def cache_reference_orbit(cx_dec, cy_dec, pw_dec, max_iter, ref_re, ref_im, ref_len,
                          fractal_type=0, julia_cx=0.0, julia_cy=0.0,
                          gen_n=3, gen_kr=0.25, gen_ki=1.0, is_floatexp=False):
    """Insert an orbit at the front of the 16-entry LRU (math_core/high_precision.py:893-916)."""
    with _ORBIT_LOCK:
        _ORBIT_CACHE.insert(0, dict(is_floatexp=is_floatexp, fractal_type=fractal_type,
                                    julia_cx=julia_cx, julia_cy=julia_cy, gen_n=gen_n,
                                    gen_kr=gen_kr, gen_ki=gen_ki, pw_dec=pw_dec, cx_dec=cx_dec,
                                    cy_dec=cy_dec, ref_len=ref_len, max_iter=max_iter,
                                    ref_re=ref_re, ref_im=ref_im))
        if len(_ORBIT_CACHE) > _CACHE_SIZE:
            _ORBIT_CACHE.pop()


PROBE_UV = [
    (0.35, 0.35), (0.65, 0.35), (0.35, 0.65), (0.65, 0.65),
    (0.5, 0.25), (0.5, 0.75), (0.25, 0.5), (0.75, 0.5),
    (0.2, 0.2), (0.8, 0.2), (0.2, 0.8), (0.8, 0.8),
    (0.5, 0.35), (0.5, 0.65), (0.35, 0.5), (0.65, 0.5),
]


def find_optimal_reference_orbit(cx_dec, cy_dec, pw_dec, ph_dec, max_iter, screen_w, screen_h,
                                 fractal_type=0, julia_cx=0.0, julia_cy=0.0,
                                 gen_n=3, gen_kr=0.25, gen_ki=1.0, is_floatexp=False, speculate=True):
    """Reference orbit for a view: cached, at the centre, or at the best of 16 probes.

    Returns (cx_dec, cy_dec, u, v, ref_re, ref_im, ref_len) where (u, v) is the
    reference's position in the view as fractions of its width and height
    (math_core/high_precision.py:919-1097).  With ``speculate`` the probe runs beside
    the centre's orbit (its work is wasted when the centre's orbit is long enough);
    without, only after it, as the reference does.  The result is the same.
    """
    ctx = decimal_context(pw_dec)
    with localcontext(ctx):
        x_min_dec = cx_dec - (pw_dec / Decimal(2))
        y_max_dec = cy_dec + (ph_dec / Decimal(2))
        best_entry, best_score = None, -1
        with _ORBIT_LOCK:
            for e in _ORBIT_CACHE:
                if e.get("is_floatexp", False) != is_floatexp:
                    continue
                if (e["fractal_type"] == fractal_type and e["julia_cx"] == julia_cx and
                        e["julia_cy"] == julia_cy and e["gen_n"] == gen_n and
                        e["gen_kr"] == gen_kr and e["gen_ki"] == gen_ki):
                    ratio = pw_dec / e["pw_dec"]
                    if Decimal("0.25") <= ratio <= Decimal("4.0"):
                        cu = float((e["cx_dec"] - x_min_dec) / pw_dec)
                        cv = float((y_max_dec - e["cy_dec"]) / ph_dec)
                        if 0.10 <= cu <= 0.90 and 0.10 <= cv <= 0.90 and e["ref_len"] > best_score:
                            best_score = e["ref_len"]
                            best_entry = e
                            if e["ref_len"] >= max_iter:
                                break
            can_reuse = False
            if best_entry is not None:
                entry_max = best_entry.get("max_iter", best_entry["ref_len"])
                natural = best_entry["ref_len"] < entry_max
                ratio = pw_dec / best_entry["pw_dec"]
                panning = Decimal("0.75") <= ratio <= Decimal("1.33")
                if best_score >= max_iter:
                    can_reuse = True
                elif panning and best_score >= 100 and (best_entry["ref_len"] >= max_iter or natural):
                    can_reuse = True
                elif natural and best_score >= int(max_iter * 0.35):
                    can_reuse = True
                elif (best_entry["cx_dec"] == cx_dec and best_entry["cy_dec"] == cy_dec and
                      best_entry["pw_dec"] == pw_dec and (best_entry["ref_len"] >= max_iter or natural)):
                    can_reuse = True
            if can_reuse and best_entry is not None:
                u = float((best_entry["cx_dec"] - x_min_dec) / pw_dec)
                v = float((y_max_dec - best_entry["cy_dec"]) / ph_dec)
                return (best_entry["cx_dec"], best_entry["cy_dec"], u, v, best_entry["ref_re"],
                        best_entry["ref_im"], min(best_entry["ref_len"], max_iter))

        bits = compute_required_prec_bits(pw_dec)
        # The probe of 16 candidates (needed when the centre's orbit escapes before
        # 0.6 max_iter, the usual case deep in a zoom) runs beside the centre's orbit,
        # and each candidate keeps its certified orbit, so the winner is not iterated
        # twice.  Results and choice are those of the sequential reference.
        # Every orbit is two native runs (two precisions, certified against each
        # other); each run is a task of its own, so the cores share the 34 runs evenly.
        pool = _probe_pool()
        args = (max_iter, fractal_type, julia_cx, julia_cy, bits, gen_n, gen_kr, gen_ki)
        centre = _Runs(pool, cx_dec, cy_dec, *args)
        probes = []

        def submit_probes():
            for (u, v) in PROBE_UV:
                with localcontext(ctx):
                    cand_x = x_min_dec + Decimal(str(u)) * pw_dec
                    cand_y = y_max_dec - Decimal(str(v)) * ph_dec
                probes.append((_Runs(pool, cand_x, cand_y, *args), cand_x, cand_y, u, v))

        may_probe = pw_dec >= Decimal("1e-10000")
        if may_probe and speculate:
            submit_probes()
        ref_re, ref_im, ref_len = _certified_orbit(*centre.result(), cx_dec, cy_dec, *args)
        best_cx, best_cy, best_u, best_v = cx_dec, cy_dec, 0.5, 0.5

        if ref_len < int(max_iter * 0.6) and may_probe:
            if not probes:
                submit_probes()
            best_esc = max(int(ref_len * 1.2), ref_len + 32)
            cand, cand_orbit = (cx_dec, cy_dec, 0.5, 0.5), None
            for runs, cand_x, cand_y, u, v in probes:
                esc, orbit = _certified_probe(*runs.result(), cand_x, cand_y, *args)
                if esc > best_esc:
                    best_esc = esc
                    cand, cand_orbit = (cand_x, cand_y, u, v), orbit
            if cand[0] != cx_dec or cand[1] != cy_dec:
                if cand_orbit is None:
                    cand_orbit = compute_single_highprec_orbit(
                        cand[0], cand[1], max_iter, fractal_type, julia_cx, julia_cy, bits,
                        gen_n=gen_n, gen_kr=gen_kr, gen_ki=gen_ki)
                c_re, c_im, c_len = cand_orbit
                if c_len > ref_len:
                    ref_re, ref_im, ref_len = c_re, c_im, c_len
                    best_cx, best_cy, best_u, best_v = cand
        else:
            for runs, *_ in probes:
                runs.cancel()  # not needed: drop those not started

        if can_reuse and best_entry is not None and best_entry["ref_len"] > ref_len:
            u = float((best_entry["cx_dec"] - x_min_dec) / pw_dec)
            v = float((y_max_dec - best_entry["cy_dec"]) / ph_dec)
            return (best_entry["cx_dec"], best_entry["cy_dec"], u, v, best_entry["ref_re"],
                    best_entry["ref_im"], min(best_entry["ref_len"], max_iter))

        cache_reference_orbit(best_cx, best_cy, pw_dec, max_iter, ref_re, ref_im, ref_len,
                              fractal_type, julia_cx, julia_cy, gen_n, gen_kr, gen_ki, is_floatexp)
        return best_cx, best_cy, best_u, best_v, ref_re, ref_im, ref_len
