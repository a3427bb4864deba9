// ap_decimal.cu -- decimal floating point on the host: the escape iteration of a
// point in the arithmetic of Python's decimal module.
//
// Orbits that the two fixed-point precisions of ap_reference_orbit cannot certify
// (bounded chaotic ones) must be iterated exactly as the reference iterates them:
// in Decimal at P = int(bits / 3.32) + 30 significant digits, every +, - and *
// rounded to P digits, half to even (math_core/high_precision.py:581-703).  This is
// that arithmetic for finite values, natively and without the Python lock, so the
// fallbacks of several threads run side by side.
//
// A value is (-1)^neg * coef * 10^exp; coef is held in base-1e8 limbs (one per
// uint64, little-endian).  Every operation forms the exact result, then rounds it;
// operands keep all their digits (inputs may carry more than P), as Decimal's do.
// Results only depend on values, never on the representation's trailing zeros.
#include <cstdint>
#include <cstring>

#include "ap_common.cuh"

namespace {

constexpr uint64_t kBase = 100000000ull;  // 1e8
constexpr int kBaseDigits = 8;
constexpr int kMaxLimbs = 400;            // 3200 digits: products of two 1600-digit operands

const uint64_t kPow10[9] = {1ull, 10ull, 100ull, 1000ull, 10000ull, 100000ull, 1000000ull,
                            10000000ull, 100000000ull};

struct Dec {
    int neg = 0;
    int64_t exp = 0;
    int n = 1;
    uint64_t d[kMaxLimbs];
};

inline bool is_zero(const Dec& a) { return a.n == 1 && a.d[0] == 0; }

inline void copy(Dec& dst, const Dec& src) {  // header and the used limbs only
    if (&dst == &src) return;
    dst.neg = src.neg;
    dst.exp = src.exp;
    dst.n = src.n;
    std::memcpy(dst.d, src.d, sizeof(uint64_t) * src.n);
}

inline void trim(Dec& a) {
    while (a.n > 1 && a.d[a.n - 1] == 0) --a.n;
}

inline int ndig8(uint64_t x) {  // digits of a limb value (0 counts as 1)
    int c = 1;
    while (c < 9 && x >= kPow10[c]) ++c;
    return c;
}

inline int64_t digits(const Dec& a) { return (int64_t)kBaseDigits * (a.n - 1) + ndig8(a.d[a.n - 1]); }

// coef = floor(coef / 10^k) for 1 <= k <= 7; the divisor is a compile-time constant,
// so no hardware division runs
template <uint64_t kDiv>
inline void div_limbs(Dec& a) {
    uint64_t rem = 0;
    for (int i = a.n - 1; i >= 0; --i) {
        const uint64_t cur = rem * kBase + a.d[i];
        const uint64_t q = cur / kDiv;
        rem = cur - q * kDiv;
        a.d[i] = q;
    }
}

// coef = floor(coef / 10^r), exp += r
void shift_right(Dec& a, int64_t r) {
    if (r <= 0) return;
    const int64_t whole = r / kBaseDigits;
    const int part = (int)(r % kBaseDigits);
    if (whole >= a.n) {
        a.n = 1;
        a.d[0] = 0;
    } else if (whole > 0) {
        std::memmove(a.d, a.d + whole, sizeof(uint64_t) * (a.n - whole));
        a.n -= (int)whole;
    }
    switch (part) {
    case 1: div_limbs<10ull>(a); break;
    case 2: div_limbs<100ull>(a); break;
    case 3: div_limbs<1000ull>(a); break;
    case 4: div_limbs<10000ull>(a); break;
    case 5: div_limbs<100000ull>(a); break;
    case 6: div_limbs<1000000ull>(a); break;
    case 7: div_limbs<10000000ull>(a); break;
    default: break;
    }
    if (part) trim(a);
    a.exp += r;
}

// coef *= 10^r (r >= 0), exact
bool shift_left(Dec& a, int64_t r) {
    if (r <= 0 || is_zero(a)) {
        if (r > 0) a.exp -= r;
        return true;
    }
    const int64_t whole = r / kBaseDigits;
    const int part = (int)(r % kBaseDigits);
    if (part) {
        const uint64_t p = kPow10[part];
        uint64_t carry = 0;
        for (int i = 0; i < a.n; ++i) {
            const uint64_t cur = a.d[i] * p + carry;
            a.d[i] = cur % kBase;
            carry = cur / kBase;
        }
        if (carry) {
            if (a.n >= kMaxLimbs) return false;
            a.d[a.n++] = carry;
        }
    }
    if (whole) {
        if (a.n + whole > kMaxLimbs) return false;
        std::memmove(a.d + whole, a.d, sizeof(uint64_t) * a.n);
        std::memset(a.d, 0, sizeof(uint64_t) * whole);
        a.n += (int)whole;
    }
    a.exp -= r;
    return true;
}

// Round to P significant digits, half to even.
void round_p(Dec& a, int P) {
    if (is_zero(a)) return;
    const int64_t D = digits(a);
    if (D <= P) return;
    const int64_t r = D - P;
    const int64_t pos = r - 1;  // the most significant dropped digit
    const int li = (int)(pos / kBaseDigits), di = (int)(pos % kBaseDigits);
    const uint64_t top = (a.d[li] / kPow10[di]) % 10;
    bool sticky = (a.d[li] % kPow10[di]) != 0;
    for (int i = 0; i < li && !sticky; ++i) sticky = a.d[i] != 0;
    shift_right(a, r);
    const bool odd = a.d[0] & 1;
    if (top > 5 || (top == 5 && (sticky || odd))) {
        uint64_t carry = 1;
        for (int i = 0; i < a.n && carry; ++i) {
            a.d[i] += carry;
            carry = a.d[i] / kBase;
            a.d[i] %= kBase;
        }
        if (carry) a.d[a.n++] = carry;
        if (digits(a) > P) shift_right(a, 1);  // 10^P: the dropped digit is 0
    }
}

int cmp_mag(const Dec& a, const Dec& b) {  // |a| vs |b| as values
    if (is_zero(a) || is_zero(b)) return is_zero(a) ? (is_zero(b) ? 0 : -1) : 1;
    const int64_t ta = a.exp + digits(a), tb = b.exp + digits(b);
    if (ta != tb) return ta < tb ? -1 : 1;
    // same leading position: compare digit by digit from the top
    static thread_local Dec x, y;
    copy(x, a);
    copy(y, b);
    const int64_t e = x.exp < y.exp ? x.exp : y.exp;
    shift_left(x, x.exp - e);
    shift_left(y, y.exp - e);
    if (x.n != y.n) return x.n < y.n ? -1 : 1;
    for (int i = x.n - 1; i >= 0; --i)
        if (x.d[i] != y.d[i]) return x.d[i] < y.d[i] ? -1 : 1;
    return 0;
}

int cmp(const Dec& a, const Dec& b) {
    const int sa = is_zero(a) ? 0 : (a.neg ? -1 : 1), sb = is_zero(b) ? 0 : (b.neg ? -1 : 1);
    if (sa != sb) return sa < sb ? -1 : 1;
    if (sa == 0) return 0;
    const int m = cmp_mag(a, b);
    return sa > 0 ? m : -m;
}

// r = a * b rounded (r must not alias a or b)
bool mul(Dec& r, const Dec& a, const Dec& b, int P) {
    if (a.n + b.n > kMaxLimbs) return false;
    r.neg = a.neg ^ b.neg;
    r.exp = a.exp + b.exp;
    const int n = a.n + b.n;
    uint64_t carry = 0;
    for (int col = 0; col < n; ++col) {
        uint64_t s = carry;
        const int i0 = col - (b.n - 1) > 0 ? col - (b.n - 1) : 0;
        const int i1 = col < a.n - 1 ? col : a.n - 1;
        // column sums stay below 2^64: at most 400 products below 1e16, plus the carry
        for (int i = i0; i <= i1; ++i) s += a.d[i] * b.d[col - i];
        r.d[col] = s % kBase;
        carry = s / kBase;
    }
    r.n = n;
    while (carry) {
        if (r.n >= kMaxLimbs) return false;
        r.d[r.n++] = carry % kBase;
        carry /= kBase;
    }
    trim(r);
    round_p(r, P);
    return true;
}

// r = a + (-1)^negate_b b rounded (r may alias a or b)
bool add(Dec& r, const Dec& a, const Dec& b0, bool negate_b, int P) {
    static thread_local Dec x, y;
    copy(x, a);
    copy(y, b0);
    if (negate_b) y.neg ^= 1;
    if (is_zero(x) || is_zero(y)) {
        if (is_zero(x) && is_zero(y)) {
            copy(r, x);
            r.neg = (x.neg && y.neg) ? 1 : 0;
            r.exp = x.exp < y.exp ? x.exp : y.exp;
            return true;
        }
        copy(r, is_zero(x) ? y : x);
        round_p(r, P);
        return true;
    }
    // an operand entirely below the result's rounding position (by a margin) acts only
    // through its sign: replace it by one unit further down
    const int64_t hx = x.exp + digits(x), hy = y.exp + digits(y);
    const int64_t top = hx > hy ? hx : hy;
    Dec* small = hx < hy ? &x : &y;
    const Dec* large = hx < hy ? &y : &x;
    int64_t cutoff = top - P - 3;
    if (large->exp < cutoff) cutoff = large->exp;
    if (small->exp + digits(*small) <= cutoff) {
        small->n = 1;
        small->d[0] = 1;
        small->exp = cutoff - 1;
    }
    const int64_t e = x.exp < y.exp ? x.exp : y.exp;
    if (!shift_left(x, x.exp - e) || !shift_left(y, y.exp - e)) return false;
    const int n = x.n > y.n ? x.n : y.n;
    for (int i = x.n; i < n; ++i) x.d[i] = 0;
    for (int i = y.n; i < n; ++i) y.d[i] = 0;
    r.exp = e;
    if (x.neg == y.neg) {
        uint64_t carry = 0;
        for (int i = 0; i < n; ++i) {
            const uint64_t s = x.d[i] + y.d[i] + carry;
            r.d[i] = s % kBase;
            carry = s / kBase;
        }
        r.n = n;
        if (carry) {
            if (r.n >= kMaxLimbs) return false;
            r.d[r.n++] = carry;
        }
        r.neg = x.neg;
    } else {
        // |x| - |y| or |y| - |x|
        int c = 0;
        for (int i = n - 1; i >= 0 && !c; --i)
            if (x.d[i] != y.d[i]) c = x.d[i] < y.d[i] ? -1 : 1;
        const Dec& p = c >= 0 ? x : y;  // r may alias a or b, not x or y
        const Dec& q = c >= 0 ? y : x;
        uint64_t borrow = 0;
        for (int i = 0; i < n; ++i) {
            const uint64_t sub = q.d[i] + borrow;
            if (p.d[i] >= sub) {
                r.d[i] = p.d[i] - sub;
                borrow = 0;
            } else {
                r.d[i] = p.d[i] + kBase - sub;
                borrow = 1;
            }
        }
        r.n = n;
        r.neg = c == 0 ? 0 : p.neg;  // x + (-x) = +0
    }
    trim(r);
    round_p(r, P);
    return true;
}

void load(Dec& a, const int64_t* meta, const uint64_t* limbs) {  // meta: neg, exp, n
    a.neg = (int)meta[0];
    a.exp = meta[1];
    a.n = (int)meta[2];
    std::memcpy(a.d, limbs, sizeof(uint64_t) * a.n);
    trim(a);
}

}  // namespace

extern "C" int ap_decimal_escape(const int64_t* meta, const uint64_t* limbs, int32_t limb_stride,
                                 int32_t prec, int32_t fractal_type, int32_t gen_n, int32_t max_iter,
                                 int32_t* k_out, int64_t* mag2_meta, uint64_t* mag2_limbs) {
    if (!meta || !limbs || !k_out || !mag2_meta || !mag2_limbs || prec < 1 || prec > 1500 ||
        limb_stride < 1 || limb_stride > kMaxLimbs / 2 || fractal_type < 0 || fractal_type > 4 ||
        (fractal_type == 4 && (gen_n < 1 || gen_n > 64)) || max_iter < 0) {
        ap::set_error("ap_decimal_escape: bad arguments");
        return AP_E_INVALID;
    }
    for (int q = 0; q < 6; ++q) {
        if (meta[3 * q + 2] < 1 || meta[3 * q + 2] > limb_stride) {
            ap::set_error("ap_decimal_escape: operand %d has %lld limbs (1..%d)", q,
                          (long long)meta[3 * q + 2], limb_stride);
            return AP_E_INVALID;
        }
    }
    const int P = prec;
    // inputs: z0_re, z0_im, c_re, c_im, k_re, k_im (exact, any number of digits)
    static thread_local Dec v[16];
    Dec &zx = v[0], &zy = v[1], &cx = v[2], &cy = v[3], &kr = v[4], &ki = v[5];
    Dec &zx2 = v[6], &zy2 = v[7], &mag = v[8], &t0 = v[9], &t1 = v[10], &t2 = v[11];
    Dec &nr = v[12], &ni = v[13], &two = v[14], &bail = v[15];
    load(zx, meta, limbs);
    load(zy, meta + 3, limbs + limb_stride);
    load(cx, meta + 6, limbs + 2 * limb_stride);
    load(cy, meta + 9, limbs + 3 * limb_stride);
    load(kr, meta + 12, limbs + 4 * limb_stride);
    load(ki, meta + 15, limbs + 5 * limb_stride);
    two.neg = 0; two.exp = 0; two.n = 1; two.d[0] = 2;
    bail.neg = 0; bail.exp = 0; bail.n = 1; bail.d[0] = 65536;
    bool ok = true;
    int k = 0;
    for (; k < max_iter && ok; ++k) {
        ok &= mul(zx2, zx, zx, P) && mul(zy2, zy, zy, P) && add(mag, zx2, zy2, false, P);
        if (!ok) break;
        if (cmp(mag, bail) > 0) break;
        if (fractal_type == 0 || fractal_type == 2) {        // zy = two*zx*zy + cy; zx = zx2 - zy2 + cx
            ok &= mul(t0, two, zx, P) && mul(t1, t0, zy, P) && add(zy, t1, cy, false, P);
            ok &= add(t2, zx2, zy2, true, P) && add(zx, t2, cx, false, P);
        } else if (fractal_type == 1 || fractal_type == 3) { // zy = two*|zx|*|zy| - cy
            copy(t2, zx);
            t2.neg = 0;
            round_p(t2, P);  // abs() rounds to the context
            ok &= mul(t0, two, t2, P);
            copy(t2, zy);
            t2.neg = 0;
            round_p(t2, P);
            ok &= mul(t1, t0, t2, P) && add(zy, t1, cy, true, P);
            ok &= add(t2, zx2, zy2, true, P) && add(zx, t2, cx, false, P);
        } else {                                             // z^n + k z + c
            copy(nr, zx);
            copy(ni, zy);
            for (int t = 0; t < gen_n - 1 && ok; ++t) {
                ok &= mul(t0, nr, zx, P) && mul(t1, ni, zy, P) && add(t2, t0, t1, true, P);  // next_r
                ok &= mul(t0, nr, zy, P) && mul(t1, ni, zx, P) && add(ni, t0, t1, false, P); // next_i
                copy(nr, t2);
            }
            Dec& kzr = zx2;  // zx2, zy2 are not needed any more in this step
            Dec& kzi = zy2;
            ok &= mul(t0, kr, zx, P) && mul(t1, ki, zy, P) && add(kzr, t0, t1, true, P);
            ok &= mul(t0, kr, zy, P) && mul(t1, ki, zx, P) && add(kzi, t0, t1, false, P);
            ok &= add(t0, nr, kzr, false, P) && add(zx, t0, cx, false, P);
            ok &= add(t1, ni, kzi, false, P) && add(zy, t1, cy, false, P);
        }
    }
    if (!ok) {
        ap::set_error("ap_decimal_escape: operand too long for %d limbs", kMaxLimbs);
        return AP_E_INVALID;
    }
    *k_out = k;
    mag2_meta[0] = mag.neg;
    mag2_meta[1] = mag.exp;
    mag2_meta[2] = mag.n;
    std::memcpy(mag2_limbs, mag.d, sizeof(uint64_t) * mag.n);
    return AP_OK;
}

// One operation of the arithmetic above (op 0: a + b, 1: a - b, 2: a * b, 3: compare
// a with b, result -1/0/1 in *cmp_out), for checking it against the decimal module.
extern "C" int ap_decimal_arith(int32_t op, const int64_t* a_meta, const uint64_t* a_limbs,
                                const int64_t* b_meta, const uint64_t* b_limbs, int32_t prec,
                                int64_t* out_meta, uint64_t* out_limbs, int32_t* cmp_out) {
    if (!a_meta || !a_limbs || !b_meta || !b_limbs || op < 0 || op > 3 || prec < 1 || prec > 1500 ||
        a_meta[2] < 1 || a_meta[2] > kMaxLimbs / 2 || b_meta[2] < 1 || b_meta[2] > kMaxLimbs / 2 ||
        (op < 3 && (!out_meta || !out_limbs)) || (op == 3 && !cmp_out)) {
        ap::set_error("ap_decimal_arith: bad arguments");
        return AP_E_INVALID;
    }
    static thread_local Dec a, b, r;
    load(a, a_meta, a_limbs);
    load(b, b_meta, b_limbs);
    if (op == 3) {
        *cmp_out = cmp(a, b);
        return AP_OK;
    }
    const bool ok = op == 2 ? mul(r, a, b, prec) : add(r, a, b, op == 1, prec);
    if (!ok) {
        ap::set_error("ap_decimal_arith: operand too long");
        return AP_E_INVALID;
    }
    out_meta[0] = r.neg;
    out_meta[1] = r.exp;
    out_meta[2] = r.n;
    std::memcpy(out_limbs, r.d, sizeof(uint64_t) * r.n);
    return AP_OK;
}
