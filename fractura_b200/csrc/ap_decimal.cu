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
#include <cmath>
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

// The iteration state of one point: z, c, K and the scratch of a step.
struct Orbit {
    Dec zx, zy, cx, cy, kr, ki, zx2, zy2, mag, t0, t1, t2, nr, ni, two, bail;
};

bool load_seeds(Orbit& o, const int64_t* meta, const uint64_t* limbs, int stride) {
    for (int q = 0; q < 6; ++q)
        if (meta[3 * q + 2] < 1 || meta[3 * q + 2] > stride) {
            ap::set_error("decimal iteration: operand %d has %lld limbs (1..%d)", q, (long long)meta[3 * q + 2],
                          stride);
            return false;
        }
    load(o.zx, meta, limbs);
    load(o.zy, meta + 3, limbs + stride);
    load(o.cx, meta + 6, limbs + 2 * stride);
    load(o.cy, meta + 9, limbs + 3 * stride);
    load(o.kr, meta + 12, limbs + 4 * stride);
    load(o.ki, meta + 15, limbs + 5 * stride);
    o.two.neg = 0; o.two.exp = 0; o.two.n = 1; o.two.d[0] = 2;
    o.bail.neg = 0; o.bail.exp = 0; o.bail.n = 1; o.bail.d[0] = 65536;
    return true;
}

// zx2, zy2 = zx^2, zy^2 and mag = zx2 + zy2 (the bailout test's operand)
bool squares(Orbit& o, int P) {
    return mul(o.zx2, o.zx, o.zx, P) && mul(o.zy2, o.zy, o.zy, P) && add(o.mag, o.zx2, o.zy2, false, P);
}

// z <- f(z) in the reference's operation order (math_core/high_precision.py:660-700),
// from z and its squares
bool step(Orbit& o, int fractal_type, int gen_n, int P) {
    bool ok = true;
    if (fractal_type == 0 || fractal_type == 2) {        // zy = two*zx*zy + cy; zx = zx2 - zy2 + cx
        ok &= mul(o.t0, o.two, o.zx, P) && mul(o.t1, o.t0, o.zy, P) && add(o.zy, o.t1, o.cy, false, P);
        ok &= add(o.t2, o.zx2, o.zy2, true, P) && add(o.zx, o.t2, o.cx, false, P);
    } else if (fractal_type == 1 || fractal_type == 3) { // zy = two*|zx|*|zy| - cy
        copy(o.t2, o.zx);
        o.t2.neg = 0;
        round_p(o.t2, P);  // abs() rounds to the context
        ok &= mul(o.t0, o.two, o.t2, P);
        copy(o.t2, o.zy);
        o.t2.neg = 0;
        round_p(o.t2, P);
        ok &= mul(o.t1, o.t0, o.t2, P) && add(o.zy, o.t1, o.cy, true, P);
        ok &= add(o.t2, o.zx2, o.zy2, true, P) && add(o.zx, o.t2, o.cx, false, P);
    } else {                                             // z^n + K z + c
        copy(o.nr, o.zx);
        copy(o.ni, o.zy);
        for (int t = 0; t < gen_n - 1 && ok; ++t) {
            ok &= mul(o.t0, o.nr, o.zx, P) && mul(o.t1, o.ni, o.zy, P) && add(o.t2, o.t0, o.t1, true, P);
            ok &= mul(o.t0, o.nr, o.zy, P) && mul(o.t1, o.ni, o.zx, P) && add(o.ni, o.t0, o.t1, false, P);
            copy(o.nr, o.t2);
        }
        Dec& kzr = o.zx2;  // the squares are not needed any more in this step
        Dec& kzi = o.zy2;
        ok &= mul(o.t0, o.kr, o.zx, P) && mul(o.t1, o.ki, o.zy, P) && add(kzr, o.t0, o.t1, true, P);
        ok &= mul(o.t0, o.kr, o.zy, P) && mul(o.t1, o.ki, o.zx, P) && add(kzi, o.t0, o.t1, false, P);
        ok &= add(o.t0, o.nr, kzr, false, P) && add(o.zx, o.t0, o.cx, false, P);
        ok &= add(o.t1, o.ni, kzi, false, P) && add(o.zy, o.t1, o.cy, false, P);
    }
    return ok;
}

// ---------------------------------------------------------------- to float64
// float(Decimal) is the correctly rounded double (CPython converts the decimal
// string).  Here: the top 36 digits T (and whether any digit below is nonzero)
// bound the value in [T, T + 1) 10^q; with a 256-bit lower bound M 2^-S of 10^q
// the value lies in [T M, (T + s) (M + 4|q| + 4)] 2^-S (s = 1 when digits were dropped).  When both ends round to the same double, so
// does the value; otherwise (a tie, or a value within ~2^-110 of one) the caller
// takes the decimal module's conversion.  (The table's lower bounds lose at most
// 2^-254 relative per power of ten, so 10^q 2^S lies in [M, M + 4|q| + 4].)

using u128 = unsigned __int128;
constexpr int kPowMax = 420;  // 10^-q for q <= 420: every normal double's range

struct Pow10Table {
    uint64_t m[kPowMax + 1][4];
    int s[kPowMax + 1];
    Pow10Table() {
        uint64_t cur[4] = {0, 0, 0, 1ull << 63};  // 2^255: 10^0 = 2^255 2^-255
        int S = 255;
        for (int q = 0; q <= kPowMax; ++q) {
            std::memcpy(m[q], cur, sizeof cur);
            s[q] = S;
            // next = cur * 16 / 10, renormalised to [2^255, 2^256), truncated (a lower bound)
            uint64_t w[5] = {cur[0] << 4, (cur[1] << 4) | (cur[0] >> 60), (cur[2] << 4) | (cur[1] >> 60),
                             (cur[3] << 4) | (cur[2] >> 60), cur[3] >> 60};
            u128 rem = 0;
            for (int i = 4; i >= 0; --i) {
                const u128 x = (rem << 64) | w[i];
                w[i] = (uint64_t)(x / 10);
                rem = x % 10;
            }
            S += 4;
            if (w[4]) {  // 2^256 <= value: drop one bit
                for (int i = 0; i < 4; ++i) w[i] = (w[i] >> 1) | (w[i + 1] << 63);
                S -= 1;
            }
            std::memcpy(cur, w, sizeof cur);
        }
    }
};

const Pow10Table& pow10_table() {
    static const Pow10Table t;  // built once (thread-safe initialisation)
    return t;
}

int bitlen(const uint64_t* x, int n) {
    for (int i = n - 1; i >= 0; --i)
        if (x[i]) return 64 * i + 64 - __builtin_clzll(x[i]);
    return 0;
}

inline int bit(const uint64_t* x, int i) { return (int)((x[i >> 6] >> (i & 63)) & 1); }

// bits [lo, lo + count) of X (count <= 64, lo >= 0, inside n limbs)
inline uint64_t bits_at(const uint64_t* x, int n, int lo, int count) {
    const int li = lo >> 6, sh = lo & 63;
    uint64_t w = x[li] >> sh;
    if (sh && li + 1 < n) w |= x[li + 1] << (64 - sh);
    return count == 64 ? w : (w & ((1ull << count) - 1));
}

// any of bits [0, k) of X set
inline bool any_below(const uint64_t* x, int k) {
    const int full = k >> 6;
    for (int i = 0; i < full; ++i)
        if (x[i]) return true;
    const int rest = k & 63;
    return rest && (x[full] & ((1ull << rest) - 1));
}

// Round X 2^-S (X: n limbs) to the nearest double, half to even; false outside the
// normal range.
bool round_to_double(const uint64_t* x, int n, int S, double* out) {
    const int b = bitlen(x, n);
    if (b == 0) {
        *out = 0.0;
        return true;
    }
    const int e2 = b - 1 - S;
    if (e2 < -1022 || e2 > 1023) return false;
    if (b <= 53) {  // exact
        *out = std::ldexp((double)x[0], -S);
        return true;
    }
    int shift = b - 53;  // the mantissa's unit is 2^(shift - S)
    uint64_t m = bits_at(x, n, shift, 53);
    const int r = bit(x, shift - 1);
    const bool sticky = any_below(x, shift - 1);
    if (r && (sticky || (m & 1))) {
        ++m;
        if (m == (1ull << 53)) {
            m >>= 1;
            ++shift;
        }
    }
    *out = std::ldexp((double)m, shift - S);
    return true;
}

// a -> float64 as float(Decimal) gives it; false when the bounds do not decide.
bool to_double(const Dec& a, double* out) {
    if (is_zero(a)) {
        *out = a.neg ? -0.0 : 0.0;
        return true;
    }
    static thread_local Dec t;
    copy(t, a);
    const int64_t D = digits(t);
    const int64_t drop = D > 36 ? D - 36 : 0;
    bool sticky = false;
    if (drop) {
        const int64_t pos = drop - 1;
        const int li = (int)(pos / kBaseDigits), di = (int)(pos % kBaseDigits);
        sticky = (t.d[li] % (kPow10[di] * 10)) != 0;
        for (int i = 0; i < li && !sticky; ++i) sticky = t.d[i] != 0;
        shift_right(t, drop);
    }
    u128 T = 0;
    for (int i = t.n - 1; i >= 0; --i) T = T * kBase + t.d[i];
    const int64_t q = t.exp;
    const uint64_t sgn = sticky ? 1 : 0;
    double lo, hi;
    if (q >= 0) {
        u128 N = T;
        for (int64_t i = 0; i < q; ++i) {
            if (N > (~(u128)0) / 20) return false;
            N *= 10;
        }
        const uint64_t x[2] = {(uint64_t)N, (uint64_t)(N >> 64)};
        const u128 N1 = N + (sticky ? 1 : 0);
        const uint64_t y[2] = {(uint64_t)N1, (uint64_t)(N1 >> 64)};
        if (!round_to_double(x, 2, 0, &lo) || !round_to_double(y, 2, 0, &hi)) return false;
    } else {
        if (-q > kPowMax) return false;
        const Pow10Table& P = pow10_table();
        const uint64_t* M = P.m[-q];
        const int S = P.s[-q];
        uint64_t L[6] = {0, 0, 0, 0, 0, 0}, U[6] = {0, 0, 0, 0, 0, 0};
        const uint64_t Tl[2] = {(uint64_t)T, (uint64_t)(T >> 64)};
        const u128 T1 = T + sgn;
        const uint64_t Tu[2] = {(uint64_t)T1, (uint64_t)(T1 >> 64)};
        // M + 4|q| + 4: the table's truncations add at most 2^-254 relative per power
        uint64_t Mu[4];
        std::memcpy(Mu, M, sizeof Mu);
        u128 c = (u128)Mu[0] + (uint64_t)(4 * (-q) + 4);
        Mu[0] = (uint64_t)c;
        for (int i = 1; i < 4 && (c >> 64); ++i) {
            c = (u128)Mu[i] + 1;
            Mu[i] = (uint64_t)c;
        }
        for (int i = 0; i < 2; ++i) {
            u128 carry = 0;
            for (int j = 0; j < 4; ++j) {
                const u128 pl = (u128)Tl[i] * M[j] + L[i + j] + carry;
                L[i + j] = (uint64_t)pl;
                carry = pl >> 64;
            }
            L[i + 4] += (uint64_t)carry;
            carry = 0;
            for (int j = 0; j < 4; ++j) {
                const u128 pu = (u128)Tu[i] * Mu[j] + U[i + j] + carry;
                U[i + j] = (uint64_t)pu;
                carry = pu >> 64;
            }
            U[i + 4] += (uint64_t)carry;
        }
        if (!round_to_double(L, 6, S, &lo) || !round_to_double(U, 6, S, &hi)) return false;
    }
    if (lo != hi) return false;
    *out = a.neg ? -lo : lo;
    return true;
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
    static thread_local Orbit o;
    if (!load_seeds(o, meta, limbs, limb_stride)) return AP_E_INVALID;
    bool ok = true;
    int k = 0;
    for (; k < max_iter; ++k) {
        if (!(ok = squares(o, prec))) break;
        if (cmp(o.mag, o.bail) > 0) break;
        if (!(ok = step(o, fractal_type, gen_n, prec))) break;
    }
    if (!ok) {
        ap::set_error("ap_decimal_escape: operand too long for %d limbs", kMaxLimbs);
        return AP_E_INVALID;
    }
    *k_out = k;
    mag2_meta[0] = o.mag.neg;
    mag2_meta[1] = o.mag.exp;
    mag2_meta[2] = o.mag.n;
    std::memcpy(mag2_limbs, o.mag.d, sizeof(uint64_t) * o.mag.n);
    return AP_OK;
}

// The orbit loop of the Decimal reference orbit (decimal_orbit: the reference's
// Decimal iteration, math_core/high_precision.py:706-875): ref_re/ref_im (max_iter + 1
// float64) receive float(Z_k); *ref_len = the escape step or max_iter; for Mandelbrot
// and its Julia set an exactly repeating orbit found at power-of-two checkpoints has its
// cycle copied to the end.  AP_E_UNSUPPORTED when a conversion is not decided by the
// bounds (the caller then runs the decimal module's loop).
extern "C" int ap_decimal_orbit(const int64_t* meta, const uint64_t* limbs, int32_t limb_stride,
                                int32_t prec, int32_t fractal_type, int32_t gen_n, int32_t max_iter,
                                double* ref_re, double* ref_im, int32_t* ref_len) {
    if (!meta || !limbs || !ref_re || !ref_im || !ref_len || prec < 1 || prec > 1500 || limb_stride < 1 ||
        limb_stride > kMaxLimbs / 2 || fractal_type < 0 || fractal_type > 4 ||
        (fractal_type == 4 && (gen_n < 1 || gen_n > 64)) || max_iter < 0) {
        ap::set_error("ap_decimal_orbit: bad arguments");
        return AP_E_INVALID;
    }
    static thread_local Orbit o;
    static thread_local Dec sx, sy;
    if (!load_seeds(o, meta, limbs, limb_stride)) return AP_E_INVALID;
    const bool periodic = fractal_type == 0 || fractal_type == 2;
    int check_step = 8, saved_k = 0;
    copy(sx, o.zx);
    copy(sy, o.zy);
    int len = max_iter;
    for (int k = 0; k < max_iter; ++k) {
        if (!to_double(o.zx, ref_re + k) || !to_double(o.zy, ref_im + k)) {
            ap::set_error("ap_decimal_orbit: conversion not decided");
            return AP_E_UNSUPPORTED;
        }
        if (!squares(o, prec)) goto too_long;
        if (cmp(o.mag, o.bail) > 0) {
            len = k;
            break;
        }
        if (periodic) {
            if (k == check_step) {
                check_step <<= 1;
                saved_k = k;
                copy(sx, o.zx);
                copy(sy, o.zy);
            } else if (k > saved_k && cmp(o.zx, sx) == 0 && cmp(o.zy, sy) == 0) {
                const int period = k - saved_k;
                for (int j = k; j <= max_iter; ++j) {
                    ref_re[j] = ref_re[j - period];
                    ref_im[j] = ref_im[j - period];
                }
                *ref_len = max_iter;
                return AP_OK;
            }
        }
        if (!step(o, fractal_type, gen_n, prec)) goto too_long;
    }
    if (!to_double(o.zx, ref_re + len) || !to_double(o.zy, ref_im + len)) {
        ap::set_error("ap_decimal_orbit: conversion not decided");
        return AP_E_UNSUPPORTED;
    }
    *ref_len = len;
    return AP_OK;
too_long:
    ap::set_error("ap_decimal_orbit: operand too long for %d limbs", kMaxLimbs);
    return AP_E_INVALID;
}

// float(Decimal) of one value (AP_E_UNSUPPORTED when the bounds do not decide), for
// checking the conversion against the decimal module.
extern "C" int ap_decimal_to_double(const int64_t* meta, const uint64_t* limbs, double* out) {
    if (!meta || !limbs || !out || meta[2] < 1 || meta[2] > kMaxLimbs) {
        ap::set_error("ap_decimal_to_double: bad arguments");
        return AP_E_INVALID;
    }
    static thread_local Dec a;
    load(a, meta, limbs);
    if (!to_double(a, out)) {
        ap::set_error("ap_decimal_to_double: not decided");
        return AP_E_UNSUPPORTED;
    }
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
