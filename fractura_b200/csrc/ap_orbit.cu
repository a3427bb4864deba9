// ap_orbit.cu -- reference orbits in binary fixed point, on the host.
//
// The perturbation tiers need the orbit Z_0, Z_1, ... of one point at the
// precision of the view (math_core/high_precision.py:706-875 iterates it in
// Decimal with int(bits / 3.32) + 30 digits).  Here every number is a signed
// fixed-point value X / 2^F held in L little-endian 64-bit limbs (two's
// complement, F = 64 (L - I): the top I limbs are the signed integer part, wide
// enough for |Z|^2 of the first escaped Z, at most (256^n + ...)^2 for z^n).
// The caller runs two precisions that bracket the Decimal one; where both give
// the same float64 orbit, so does the Decimal iteration.
//
// Products are truncated: partial products more than two limbs below the unit
// of the last kept limb are skipped (their total is below 2^-F).  Each stored
// orbit value is rounded to float64 correctly (round half to even), as
// float(Decimal) rounds.  The loop is serial; callers run candidates of the
// 16-point probe in parallel threads.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <utility>
#include <vector>

#include "ap_common.cuh"

namespace {

using u64 = uint64_t;
using u128 = unsigned __int128;

constexpr int kMaxLimbs = 160;  // 10176 fractional bits: views down to ~1e-3000

struct Fx {  // sign-magnitude working form
    int neg;
    u64 m[kMaxLimbs];
};

inline bool is_zero(const u64* a, int L) {
    for (int i = 0; i < L; ++i)
        if (a[i]) return false;
    return true;
}

inline int cmp_mag(const u64* a, const u64* b, int L) {
    for (int i = L - 1; i >= 0; --i) {
        if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
    }
    return 0;
}

inline void add_mag(u64* r, const u64* a, const u64* b, int L) {  // r = a + b
    u64 carry = 0;
    for (int i = 0; i < L; ++i) {
        const u128 s = (u128)a[i] + b[i] + carry;
        r[i] = (u64)s;
        carry = (u64)(s >> 64);
    }
}

inline void sub_mag(u64* r, const u64* a, const u64* b, int L) {  // r = a - b, a >= b
    u64 borrow = 0;
    for (int i = 0; i < L; ++i) {
        const u128 d = (u128)a[i] - b[i] - borrow;
        r[i] = (u64)d;
        borrow = (u64)((d >> 64) & 1);
    }
}

// r = (-1)^an |a| + (-1)^bn |b| on sign-magnitude values (r may alias a or b).
inline void add_s(Fx& r, const Fx& a, int an, const Fx& b, int bn, int L) {
    if (an == bn) {
        add_mag(r.m, a.m, b.m, L);
        r.neg = an && !is_zero(r.m, L);
        return;
    }
    const int c = cmp_mag(a.m, b.m, L);
    if (c >= 0) {
        sub_mag(r.m, a.m, b.m, L);
        r.neg = c == 0 ? 0 : an;
    } else {
        sub_mag(r.m, b.m, a.m, L);
        r.neg = bn;
    }
}

inline void add(Fx& r, const Fx& a, const Fx& b, int L) { add_s(r, a, a.neg, b, b.neg, L); }
inline void sub(Fx& r, const Fx& a, const Fx& b, int L) { add_s(r, a, a.neg, b, !b.neg, L); }

// Column accumulator of the product-scanning (Comba) products below: the value is
// lo + hi * 2^64, the low and high halves of the products summed in two independent
// 128-bit sums (a column has at most 2 * kMaxLimbs products, so neither overflows).
// The carry into the next column is formed once per column, in shift().
struct Acc3 {
    u128 lo = 0, hi = 0;
    inline void add(u128 p) {
        lo += (u64)p;
        hi += (u64)(p >> 64);
    }
    inline void add_twice(const Acc3& o) {  // += 2 * o
        lo += o.lo << 1;
        hi += o.hi << 1;
    }
    inline u64 shift() {  // take the finished column, keep the rest as the carry
        const u64 out = (u64)lo;
        lo = (lo >> 64) + hi;
        hi = 0;
        return out;
    }
};

// r = a * b (fixed point, truncated).  Product limb k (of 2L) has weight
// 2^(64 k - 2F); the result keeps limbs [L - I, 2L - I).  Partial products with
// index i + j < L - I - 2 are not formed: together they are worth less than one
// unit of the last kept limb.  The kept pairs are summed column by column, so the
// result is the exact sum of the same partial products in any order of
// evaluation; columns above the kept range are not formed (nothing carries down).
inline void mul(Fx& r, const Fx& a, const Fx& b, int L, int I) {
    const int lo = L - I - 2 > 0 ? L - I - 2 : 0;
    const int keep = L - I, top = 2 * L - I - 1;
    Acc3 acc;
    for (int col = lo; col <= top; ++col) {
        const int i0 = col - (L - 1) > 0 ? col - (L - 1) : 0;
        const int i1 = col < L - 1 ? col : L - 1;
        for (int i = i0; i <= i1; ++i) acc.add((u128)a.m[i] * b.m[col - i]);
        const u64 limb = acc.shift();
        if (col >= keep) r.m[col - keep] = limb;
    }
    r.neg = (a.neg ^ b.neg) && !is_zero(r.m, L);
}

// r = a * a: the same column sums as mul(r, a, a), each symmetric pair formed once
// (summed apart, then added twice).
inline void sqr(Fx& r, const Fx& a, int L, int I) {
    const int lo = L - I - 2 > 0 ? L - I - 2 : 0;
    const int keep = L - I, top = 2 * L - I - 1;
    Acc3 acc;
    for (int col = lo; col <= top; ++col) {
        const int i0 = col - (L - 1) > 0 ? col - (L - 1) : 0;
        Acc3 off;
        for (int i = i0; 2 * i < col; ++i) off.add((u128)a.m[i] * a.m[col - i]);
        acc.add_twice(off);
        if ((col & 1) == 0 && col / 2 < L) acc.add((u128)a.m[col / 2] * a.m[col / 2]);
        const u64 limb = acc.shift();
        if (col >= keep) r.m[col - keep] = limb;
    }
    r.neg = 0;
}

// mul and sqr with the limb counts fixed at compile time: the same partial products
// and column sums as mul / sqr, every column written out by the templates below.  An orbit picks its pair
// once (pick_products); sizes outside the table use the runtime-bound forms.
using MulFn = void (*)(Fx&, const Fx&, const Fx&);
using SqrFn = void (*)(Fx&, const Fx&);

// Column col of a product: the partial products a[i] * b[col - i] for i in [i0, i0 + n),
// one expression each (a fold over an index sequence), so every column is unrolled.
template <int COL, int I0, size_t... K>
inline void column_sum(Acc3& acc, const u64* a, const u64* b, std::index_sequence<K...>) {
    (acc.add((u128)a[I0 + (int)K] * b[COL - I0 - (int)K]), ...);
}

template <int L, int I, int COL>
inline void mul_column(Acc3& acc, const u64* a, const u64* b, u64* r) {
    constexpr int i0 = COL - (L - 1) > 0 ? COL - (L - 1) : 0;
    constexpr int i1 = COL < L - 1 ? COL : L - 1;
    column_sum<COL, i0>(acc, a, b, std::make_index_sequence<i1 - i0 + 1>{});
    const u64 limb = acc.shift();
    if constexpr (COL >= L - I) r[COL - (L - I)] = limb;
}

template <int L, int I, size_t... C>
inline void mul_columns(Acc3& acc, const u64* a, const u64* b, u64* r, std::index_sequence<C...>) {
    constexpr int lo = L - I - 2 > 0 ? L - I - 2 : 0;
    (mul_column<L, I, lo + (int)C>(acc, a, b, r), ...);
}

// Off-diagonal pairs of column col of a square (i < col - i), summed once.
template <int L, int I, int COL>
inline void sqr_column(Acc3& acc, const u64* a, u64* r) {
    constexpr int i0 = COL - (L - 1) > 0 ? COL - (L - 1) : 0;
    constexpr int n_off = (COL + 1) / 2 - i0 > 0 ? (COL + 1) / 2 - i0 : 0;  // i in [i0, ceil(col/2))
    Acc3 off;
    column_sum<COL, i0>(off, a, a, std::make_index_sequence<n_off>{});
    acc.add_twice(off);
    if constexpr ((COL & 1) == 0 && COL / 2 < L) acc.add((u128)a[COL / 2] * a[COL / 2]);
    const u64 limb = acc.shift();
    if constexpr (COL >= L - I) r[COL - (L - I)] = limb;
}

template <int L, int I, size_t... C>
inline void sqr_columns(Acc3& acc, const u64* a, u64* r, std::index_sequence<C...>) {
    constexpr int lo = L - I - 2 > 0 ? L - I - 2 : 0;
    (sqr_column<L, I, lo + (int)C>(acc, a, r), ...);
}

template <int L, int I>
void mul_fixed(Fx& r, const Fx& a, const Fx& b) {
    constexpr int lo = L - I - 2 > 0 ? L - I - 2 : 0, top = 2 * L - I - 1;
    Acc3 acc;
    mul_columns<L, I>(acc, a.m, b.m, r.m, std::make_index_sequence<top - lo + 1>{});
    r.neg = (a.neg ^ b.neg) && !is_zero(r.m, L);
}

template <int L, int I>
void sqr_fixed(Fx& r, const Fx& a) {
    constexpr int lo = L - I - 2 > 0 ? L - I - 2 : 0, top = 2 * L - I - 1;
    Acc3 acc;
    sqr_columns<L, I>(acc, a.m, r.m, std::make_index_sequence<top - lo + 1>{});
    r.neg = 0;
}

struct Products {
    MulFn mul = nullptr;
    SqrFn sqr = nullptr;
};

template <int I>
Products pick_for(int L) {
    switch (L) {
#define AP_FIXED_LIMBS(n) \
    case n: return {mul_fixed<n, I>, sqr_fixed<n, I>};
        AP_FIXED_LIMBS(3) AP_FIXED_LIMBS(4) AP_FIXED_LIMBS(5) AP_FIXED_LIMBS(6) AP_FIXED_LIMBS(7)
        AP_FIXED_LIMBS(8) AP_FIXED_LIMBS(9) AP_FIXED_LIMBS(10) AP_FIXED_LIMBS(11) AP_FIXED_LIMBS(12)
        AP_FIXED_LIMBS(13) AP_FIXED_LIMBS(14) AP_FIXED_LIMBS(15) AP_FIXED_LIMBS(16) AP_FIXED_LIMBS(17)
        AP_FIXED_LIMBS(18) AP_FIXED_LIMBS(19) AP_FIXED_LIMBS(20) AP_FIXED_LIMBS(21) AP_FIXED_LIMBS(22)
        AP_FIXED_LIMBS(23) AP_FIXED_LIMBS(24)
#undef AP_FIXED_LIMBS
    default: return {};
    }
}

Products pick_products(int L, int I) {
    if (I == 1) return pick_for<1>(L);
    if (I == 2) return pick_for<2>(L);
    return {};
}

// Correctly rounded float64 (round half to even) of a sign-magnitude value.
double to_double(const Fx& a, int L, int I) {
    int top = L - 1;
    while (top >= 0 && a.m[top] == 0) --top;
    if (top < 0) return a.neg ? -0.0 : 0.0;
    const int lz = __builtin_clzll(a.m[top]);
    const int p = 64 * top + (63 - lz);  // index of the leading one bit
    // 64-bit window with the leading bit at its top, then a sticky bit below it.
    auto bit_window = [&](int hi_bit) -> u64 {  // bits [hi_bit - 63, hi_bit]
        const int lo_bit = hi_bit - 63;
        u64 w = 0;
        if (lo_bit >= 0) {
            const int li = lo_bit >> 6, sh = lo_bit & 63;
            w = a.m[li] >> sh;
            if (sh && li + 1 < L) w |= a.m[li + 1] << (64 - sh);
        } else {
            w = a.m[0] << (-lo_bit);
        }
        return w;
    };
    const u64 win = bit_window(p);
    bool sticky = false;
    const int lo_bit = p - 63;
    if (lo_bit > 0) {
        const int li = lo_bit >> 6, sh = lo_bit & 63;
        for (int i = 0; i < li && !sticky; ++i) sticky = a.m[i] != 0;
        if (!sticky && sh) sticky = (a.m[li] & ((1ULL << sh) - 1)) != 0;
    }
    u64 mant = win >> 11;
    const u64 rest = win & 0x7FF;
    int e2 = p;
    if (rest > 0x400 || (rest == 0x400 && (sticky || (mant & 1)))) {
        ++mant;
        if (mant == (1ULL << 53)) {
            mant >>= 1;
            ++e2;
        }
    }
    const int F = 64 * (L - I);
    const double v = std::ldexp((double)mant, e2 - 52 - F);
    return a.neg ? -v : v;
}

void load(Fx& r, const u64* twos, int L) {  // two's complement limbs -> sign-magnitude
    const int neg = (twos[L - 1] >> 63) & 1;
    if (!neg) {
        std::memcpy(r.m, twos, sizeof(u64) * L);
        r.neg = 0;
        return;
    }
    u64 carry = 1;
    for (int i = 0; i < L; ++i) {
        const u128 s = (u128)(~twos[i]) + carry;
        r.m[i] = (u64)s;
        carry = (u64)(s >> 64);
    }
    r.neg = !is_zero(r.m, L);
}

inline bool equal(const Fx& a, const Fx& b, int L) {
    return a.neg == b.neg && cmp_mag(a.m, b.m, L) == 0;
}

// ---- Certification against the Decimal iteration (quadratic formulas) ----------------
// The reference iterates the orbit in Decimal with P significant digits; every operation
// rounds with relative error at most u = 5 10^-P.  The run here is fixed point with F
// fractional bits; a truncated square is off by less than 1.01 units of 2^-F (so x^2 - y^2
// by 2.02 and 2 x y = (x + y)^2 - x^2 - y^2 by 3.03), a stored seed by 0.5.  Both follow the
// same map.  In the complex modulus, z^2 moves by at most
// (2 |z| + E) E when z moves by E, and so does Burning Ship's step, whose fold
// (x, y) -> (|x|, |y|) moves no point farther; so the two runs' distance obeys
//   E_{k+1} <= (2 |z| + E_k) E_k + r_dec + r_fix,
//   r_dec <= u [2 (x^2 + y^2) + |x'| + 4 |x| |y| + |y'|] (with margins),  r_fix = 6.5 2^-F,
// where |x'| <= x^2 + y^2 + |c_x| and |y'| <= 2 |x| |y| + |c_y|, the magnitudes taken at
// the fixed-point value plus E.  The two float64 roundings of a component agree wherever
// E_k is below half its distance to the nearest float64 rounding boundary (half: the
// boundaries below a power of two are twice as dense), and the bailout decisions agree
// wherever |Z|^2 is farther from 65536 than its own error bound.  Multibrot z^n + k z + c
// grows the bound by (|z| + E)^n - |z|^n + |k| E, with the roundings of its power loop.
// E is held scaled by 2^B (u 2^B in [1, 2)), so it neither underflows nor overflows.
constexpr int kNoDist = -(1 << 30);

u64 bits_at(const Fx& a, int L, int lo_bit) {  // bits [lo_bit, lo_bit + 63]; zero outside [0, 64 L)
    if (lo_bit <= -64) return 0;
    if (lo_bit < 0) return a.m[0] << (-lo_bit);
    const int li = lo_bit >> 6, sh = lo_bit & 63;
    if (li >= L) return 0;
    u64 w = a.m[li] >> sh;
    if (sh && li + 1 < L) w |= a.m[li + 1] << (64 - sh);
    return w;
}

// floor(log2) of a lower bound on the distance from a (in value units) to the nearest
// float64 rounding boundary; kNoDist when there is none to give (zero, a value near
// the subnormal range, or 64 bits below the mantissa at the midpoint itself).
int rounding_distance_exp(const Fx& a, int L, int I) {
    int top = L - 1;
    while (top >= 0 && a.m[top] == 0) --top;
    if (top < 0) return kNoDist;
    const int p = 64 * top + (63 - __builtin_clzll(a.m[top]));
    const int F = 64 * (L - I);
    if (p - F < -1000) return kNoDist;
    const int lo_bit = p - 116;  // the 64 bits just below the mantissa's last bit
    const u64 w = bits_at(a, L, lo_bit), half = 1ULL << 63;
    const u64 d = w < half ? half - w - 1 : w - half;  // the bits below may add up to one unit
    if (d == 0) return kNoDist;
    return (63 - __builtin_clzll(d)) + lo_bit - F;
}

struct Cert {
    bool ok = false;
    int B = 0;              // scaled quantities are value * 2^B
    double u_s = 0.0;       // Decimal unit roundoff, scaled
    double r_fix_s = 0.0;   // the fixed-point run's error per step, scaled
    double E = 0.0;         // the bound on |z_Decimal - z_fixed| (complex modulus), scaled
    double cx = 0.0, cy = 0.0, cabs = 0.0, kabs = 0.0;
    double ulp_s = 0.0;     // 2^-F, scaled

    void start(int dec_digits, int L, int I, double cxd, double cyd, double krd, double kid, bool julia) {
        const double l2_10 = 3.3219280948873623478703194294894;
        ok = dec_digits > 0;
        B = (int)std::ceil((dec_digits - 1) * l2_10) + 1;
        u_s = std::exp2((double)(B - 1) - (dec_digits - 1) * l2_10) * (1.0 + 1e-9);
        const int F = 64 * (L - I);
        ulp_s = std::ldexp(1.0, B - F);
        r_fix_s = 6.5 * ulp_s;
        E = julia ? 0.75 * ulp_s : 0.0;  // a Julia orbit starts at the rounded pixel
        cx = std::fabs(cxd);
        cy = std::fabs(cyd);
        cabs = std::hypot(cxd, cyd) * (1.0 + 0x1p-48);
        kabs = std::hypot(krd, kid) * (1.0 + 0x1p-48);
    }
    // true when the float64 rounding of a is certain: the error bound is below half its
    // distance to a rounding boundary (scaled error E: E 2^-B < 2^(ilogb(E) + 1 - B))
    bool rounds_alike(const Fx& a, int L, int I, double Es) const {
        if (Es == 0.0) return true;
        if (!(Es < 1e300)) return false;
        const int dexp = rounding_distance_exp(a, L, I);
        return dexp != kNoDist && dexp >= std::ilogb(Es) + 3 - B;
    }
};

}  // namespace

static int orbit_impl(const uint64_t* seeds, int32_t limbs, int32_t int_limbs, int32_t fractal_type,
                      int32_t gen_n, int32_t max_iter, int32_t escape_only, double* ref_re, double* ref_im,
                      int32_t* ref_len, double* escape_mag2, uint64_t* trace_hash, int32_t dec_digits,
                      int32_t* certified) {
    if (certified) *certified = 0;
    if (!seeds || !ref_len || max_iter < 0 || fractal_type < 0 || fractal_type > 4 ||
        (fractal_type == 4 && (gen_n < 1 || gen_n > 64)) || (!escape_only && (!ref_re || !ref_im))) {
        ap::set_error("ap_reference_orbit: bad arguments");
        return AP_E_INVALID;
    }
    // integer bits needed: |Z|^2 of the first escaped Z (|Z_prev| <= 256) plus sign
    const int n = fractal_type == 4 ? (gen_n > 2 ? gen_n : 2) : 2;
    const int need = (16 * n + 8 + 1 + 63) / 64;
    if (int_limbs < need || limbs <= int_limbs || limbs > kMaxLimbs) {
        ap::set_error("ap_reference_orbit: %d limbs with %d integer limbs (need >= %d integer limbs, "
                      "at most %d limbs)", limbs, int_limbs, need, kMaxLimbs);
        return AP_E_INVALID;
    }
    const int L = limbs, I = int_limbs;
    const Products fixed = pick_products(L, I);
    auto MUL = [&](Fx& r, const Fx& a, const Fx& b) {
        if (fixed.mul) fixed.mul(r, a, b);
        else mul(r, a, b, L, I);
    };
    auto SQR = [&](Fx& r, const Fx& a) {
        if (fixed.sqr) fixed.sqr(r, a);
        else sqr(r, a, L, I);
    };
    // seeds: z0_re, z0_im, c_re, c_im, k_re, k_im, each L limbs
    std::vector<Fx> v(16);
    Fx &zx = v[0], &zy = v[1], &cx = v[2], &cy = v[3], &kr = v[4], &ki = v[5];
    Fx &zx2 = v[6], &zy2 = v[7], &t0 = v[8], &t1 = v[9], &t2 = v[10], &t3 = v[11];
    Fx &sx = v[12], &sy = v[13], &bail = v[14], &mag = v[15];
    load(zx, seeds, L);
    load(zy, seeds + L, L);
    load(cx, seeds + 2 * L, L);
    load(cy, seeds + 3 * L, L);
    load(kr, seeds + 4 * L, L);
    load(ki, seeds + 5 * L, L);
    std::memset(bail.m, 0, sizeof(u64) * L);
    bail.m[L - I] = 65536;
    bail.neg = 0;
    Cert cert;
    if (certified && !escape_only)
        cert.start(dec_digits, L, I, to_double(cx, L, I), to_double(cy, L, I), to_double(kr, L, I),
                   to_double(ki, L, I), fractal_type == 2 || fractal_type == 3);

    const bool periodic = (fractal_type == 0 || fractal_type == 2) && !escape_only;
    int check_step = 8, saved_k = 0;
    sx = zx;
    sy = zy;
    int len = max_iter;
    // A multiplicative hash over the float64 bits of every Z_k (xor, then multiply
    // by an odd constant: each step is a bijection of the state, so a single
    // differing value always changes the state): lets two runs at different
    // precisions confirm they followed the same float64 trajectory.
    u64 hash = 1469598103934665603ULL;
    auto mix = [&](double d) {
        u64 b;
        std::memcpy(&b, &d, 8);
        hash = (hash ^ b) * 0x9E3779B97F4A7C15ULL;
        hash ^= hash >> 29;
    };
    for (int k = 0; k < max_iter; ++k) {
        if (!escape_only || trace_hash) {
            const double re = to_double(zx, L, I), im = to_double(zy, L, I);
            if (!escape_only) {
                ref_re[k] = re;
                ref_im[k] = im;
            }
            if (trace_hash) {
                mix(re);
                mix(im);
            }
        }
        SQR(zx2, zx);
        SQR(zy2, zy);
        add(mag, zx2, zy2, L);
        const bool escaped = !mag.neg && cmp_mag(mag.m, bail.m, L) > 0;
        double Emag_s = 0.0;
        if (cert.ok) {
            // the stored values, then the bailout decision (and |Z|^2 at escape)
            const double xf = to_double(zx, L, I), yf = to_double(zy, L, I);
            const double Et = std::ldexp(cert.E, -cert.B);
            const double az = std::hypot(xf, yf) * (1.0 + 0x1p-48);  // |z| of this run, from above
            const double ax = std::fabs(xf) * (1.0 + 0x1p-50) + Et, ay = std::fabs(yf) * (1.0 + 0x1p-50) + Et;
            const double m2 = (az + Et) * (az + Et);                  // |z|^2 of either run, from above
            // |z|^2 moves by at most (2 |z| + E) E
            const double grow2 = (2.0 * az + Et) * cert.E * (1.0 + 1e-12);
            Emag_s = (grow2 + cert.u_s * 2.0001 * m2 + 2.02 * cert.ulp_s) * (1.0 + 1e-12);
            const double magf = xf * xf + yf * yf;
            const double margin = std::ldexp(Emag_s, -cert.B) + 65536.0 * 0x1p-48;
            cert.ok = cert.rounds_alike(zx, L, I, cert.E) && cert.rounds_alike(zy, L, I, cert.E) &&
                      std::fabs(magf - 65536.0) > margin;
            if (cert.ok && escaped && escape_mag2) cert.ok = cert.rounds_alike(mag, L, I, Emag_s);
            // the next step's bound
            if (fractal_type <= 3) {
                const double rdec = 2.0001 * m2 + 1.0001 * (m2 + cert.cx) + 4.0001 * ax * ay +
                                    1.0001 * (2.0 * ax * ay + cert.cy);
                cert.E = grow2 + cert.u_s * rdec * (1.0 + 1e-12) + cert.r_fix_s;
            } else {
                // z^n + k z + c moves by at most (|z| + E)^n - |z|^n + |k| E, expanded so that
                // nothing cancels: E sum_{j=1..n} C(n, j) |z|^(n-j) E^(j-1)
                const int nn = gen_n;
                double sum = 0.0, c = nn, ep = 1.0, A = az + Et, An = 1.0, geo = 0.0, aj = 1.0;
                for (int j = 1; j <= nn; ++j) {
                    sum += c * std::pow(az, nn - j) * ep;
                    c = c * (nn - j) / (j + 1);
                    ep *= Et;
                }
                for (int j = 0; j < nn; ++j) An *= A;
                for (int j = 0; j <= nn - 2; ++j) {  // 1 + |z| + ... + |z|^(n-2)
                    geo += aj;
                    aj *= az;
                }
                const double grow = (sum + cert.kabs) * cert.E * (1.0 + 1e-10);
                // the Decimal loop rounds 4 products and 2 sums per power, the k z products
                // and the final sums; the fixed-point run truncates 4 products per power (an
                // error that the later powers multiply by |z|) and 4 for k z, and carries the
                // rounded k and c
                const double rdec = (4.0004 * (nn - 1) + 2.0002) * An + 6.0006 * cert.kabs * A + 2.0002 * cert.cabs;
                const double rfix = (2.86 * (geo + 1.0) + 0.71 * (az + 1.0)) * cert.ulp_s;
                cert.E = grow + cert.u_s * rdec * (1.0 + 1e-10) + rfix * (1.0 + 1e-10);
            }
        }
        if (escaped) {
            len = k;
            if (escape_mag2) *escape_mag2 = to_double(mag, L, I);
            break;
        }
        if (periodic) {
            if (k == check_step) {
                check_step <<= 1;
                saved_k = k;
                sx = zx;
                sy = zy;
            } else if (k > saved_k && equal(zx, sx, L) && equal(zy, sy, L)) {
                const int period = k - saved_k;
                for (int j = k; j <= max_iter; ++j) {
                    ref_re[j] = ref_re[j - period];
                    ref_im[j] = ref_im[j - period];
                }
                *ref_len = max_iter;
                if (trace_hash) *trace_hash = hash;
                return AP_OK;  // a copied cycle is not certified: the caller compares two runs
            }
        }
        if (fractal_type == 0 || fractal_type == 2) {  // z^2 + c
            // 2 x y = (x + y)^2 - x^2 - y^2: a square costs about half a product
            add(t2, zx, zy, L);
            SQR(t0, t2);
            sub(t0, t0, zx2, L);
            sub(t0, t0, zy2, L);
            sub(t1, zx2, zy2, L);
            add(zx, t1, cx, L);
            add(zy, t0, cy, L);
        } else if (fractal_type == 1 || fractal_type == 3) {  // Burning Ship: 2|x||y| - c_y
            add_s(t2, zx, 0, zy, 0, L);  // |x| + |y|
            SQR(t0, t2);
            sub(t0, t0, zx2, L);
            sub(t0, t0, zy2, L);
            sub(t1, zx2, zy2, L);
            add(zx, t1, cx, L);
            sub(zy, t0, cy, L);
        } else {  // Multibrot z^n + K z + c
            Fx& nr = v[12];  // the checkpoint slots are free: no period detection here
            Fx& ni = v[13];
            nr = zx;
            ni = zy;
            for (int t = 0; t < gen_n - 1; ++t) {
                MUL(t0, nr, zx);
                MUL(t1, ni, zy);
                MUL(t2, nr, zy);
                MUL(t3, ni, zx);
                sub(nr, t0, t1, L);
                add(ni, t2, t3, L);
            }
            MUL(t0, kr, zx);
            MUL(t1, ki, zy);
            MUL(t2, kr, zy);
            MUL(t3, ki, zx);
            sub(t0, t0, t1, L);  // Re(K z)
            add(t2, t2, t3, L);  // Im(K z)
            add(t0, nr, t0, L);
            add(zx, t0, cx, L);
            add(t2, ni, t2, L);
            add(zy, t2, cy, L);
        }
    }
    if (!escape_only) {
        ref_re[len] = to_double(zx, L, I);
        ref_im[len] = to_double(zy, L, I);
    }
    *ref_len = len;
    if (trace_hash) *trace_hash = hash;
    if (certified) *certified = cert.ok ? 1 : 0;
    return AP_OK;
}

extern "C" int ap_reference_orbit(const uint64_t* seeds, int32_t limbs, int32_t int_limbs,
                                  int32_t fractal_type,
                                  int32_t gen_n, int32_t max_iter, int32_t escape_only,
                                  double* ref_re, double* ref_im, int32_t* ref_len,
                                  double* escape_mag2, uint64_t* trace_hash) {
    return orbit_impl(seeds, limbs, int_limbs, fractal_type, gen_n, max_iter, escape_only, ref_re, ref_im,
                      ref_len, escape_mag2, trace_hash, 0, nullptr);
}

extern "C" int ap_reference_orbit_cert(const uint64_t* seeds, int32_t limbs, int32_t int_limbs,
                                       int32_t fractal_type, int32_t gen_n, int32_t max_iter,
                                       int32_t dec_digits, double* ref_re, double* ref_im, int32_t* ref_len,
                                       double* escape_mag2, int32_t* certified) {
    if (!certified || dec_digits < 1) {
        ap::set_error("ap_reference_orbit_cert: bad arguments");
        return AP_E_INVALID;
    }
    return orbit_impl(seeds, limbs, int_limbs, fractal_type, gen_n, max_iter, 0, ref_re, ref_im, ref_len,
                      escape_mag2, nullptr, dec_digits, certified);
}
