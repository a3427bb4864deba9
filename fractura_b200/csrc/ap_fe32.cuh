// ap_fe32.cuh -- FP32-mantissa FloatExp perturbation (AP_TIER_FLOATEXP32): one pixel.
//
// The engine's fast form of the perturbation tiers, for all five formulas.  The
// delta is held as
//   dz = w * 2^e,  w a complex float32 with max(|w_re|, |w_im|) in [1, 2)
// after renormalisation, e an int32 exponent; delta_c = dcm * 2^-E with dcm a
// complex float32 and E the frame's exponent scale.  With S = 2^e (float, 0 below
// 2^-126) and D = dcm 2^(-E-e) (0 for the Julia sets), one step runs in FP32:
//   Mandelbrot, Julia:   w' = 2 Z w + S w^2 + D
//   Burning Ship and its Julia set (y' = 2 |x| |y| - c_y):
//     w'_x = 2 (Z_x w_x - Z_y w_y) + S (w_x^2 - w_y^2) + D_x
//     w'_y = 2 (|Z_x| d_y + |Z_y| d_x + S d_x d_y) - D_y,
//     d_x = (|Z_x + dz_x| - |Z_x|) 2^-e = s w_x when Z_x + dz_x keeps the sign s of
//     Z_x, else -s (2 Z_x 2^-e + w_x) (and d_y alike);
//   Multibrot z^n + k z + c:  P_1 = w, P_{j+1} = P_j Z + (S P_j + Z^j) w (P_j the
//     scaled (Z + dz)^j - Z^j), w' = P_n + k w + D.
// The exponent changes only when |w| leaves [2^-16, 2^16] (exact power-of-two
// rescaling, as the FP64 FloatExp tier of the reference does with its 2^16 steps,
// math_core/cuda_kernels.py:913-923; its Burning Ship and Multibrot delta steps are
// :927-1010).
//
// What stays FP64 (and how):
//   * the reference orbit: FP64 records (ap_pack_orbit) feed every FP64
//     decision; the FP32 step reads a float copy (ap_pack_fe32);
//   * BLA validity radii: r^2 * 2^B in FP64 (B a power-of-two bias so that
//     |dz|^2 * 2^B does not underflow near any radius), compared with
//     (double)|w|^2 * 2^(2e + B);
//   * the Pauldelbrot glitch test |Z + dz|^2 < 1e-6 |Z|^2, the escape test, the
//     Burning Ship sign tests and the one-pass rebase test |Z + dz| < |dz|: an FP32
//     screen decides whether each can fire at this step (a sign can change only when
//     |dz_x| >= |Z_x| / 2, a rebase only when |dz| > |Z| / 2); when it can, the test
//     is evaluated in FP64 on Z and the exactly converted delta;
//   * the smooth value at escape and the stage-2 direct iteration (after the
//     reference escapes) run in FP64.
// BLA leaps: A = am 2^ea, B = bm 2^eb with float mantissas (ap_pack_fe32);
// dz' = A dz + B dc keeps exponent e + ea.
//
// One-pass rebasing (AP_FLAG_REBASE, fractal types 0, 1, 4) as in the FP64-delta
// form: when |Z_m + dz| < |dz| or the reference has ended, dz <- Z_m + dz (formed in
// FP64, then renormalised) and m <- 0; no pixel is glitched and there is no stage 2.
//
// FP64 slow path.  Two cases leave the FP32 range and take one step (or leap)
// in FP64 on the same normalised quantities, renormalised in FP64 before the
// result is narrowed to float: steps where the reference orbit passes close to
// zero (|Z| < 2^-50: Z itself underflows in float, and 2 Z w loses its
// exponent; marked by ap_pack_fe32), and deltas whose scale is so far from
// dc's that the power-of-two factor of the dc term leaves [2^-120, 2^120].
//
// The radius bias is a constant 2^600: radii lie in [2^-1074, 1/4], so r^2 2^600
// stays finite and normal, and |dz|^2 2^600 only saturates (to 0 or inf) where
// it is far from every radius -- where the comparison's outcome is certain.
#pragma once

#include "ap_common.cuh"
#include "ap_coarse.cuh"

namespace ap {

constexpr int kRadiusBias = 600;

struct Fe32Bla {        // 32 bytes per (step, level)
    float ar, ai, br, bi;
    int ea, eb, pad0, pad1;
};

__device__ __forceinline__ float exp2i_f(int n) {  // 2^n as float: 0 below 2^-126, 2^127 above
    n = min(n, 127);
    return (n < -126) ? 0.0f : __int_as_float((n + 127) << 23);
}

__device__ __forceinline__ double exp2i_d(int n) {  // 2^n as double: 0 below 2^-1022, inf above 2^1023
    return (n < -1022) ? 0.0 : (n > 1023 ? __longlong_as_double(0x7ff0000000000000LL)
                                         : __longlong_as_double((long long)(n + 1023) << 52));
}

// Exponent of max(|x|, |y|) (floor(log2)), for non-zero finite inputs.
__device__ __forceinline__ int ilogb_max(float x, float y) {
    const float m = fmaxf(fabsf(x), fabsf(y));
    return ((__float_as_int(m) >> 23) & 0xff) - 127;
}

// Normalise a double pair into (float mantissa with max component in [1, 2), exponent
// added to e).  Zero stays zero with e unchanged.
__device__ __forceinline__ void renorm_to_float(double x, double y, float& wx, float& wy, int& e) {
    const double m = fmax(fabs(x), fabs(y));
    if (!(m > 0.0) || !isfinite(m)) {
        wx = (float)x;
        wy = (float)y;
        return;
    }
    const int ex = ilogb(m);
    const double f = ldexp(1.0, -ex);
    wx = (float)(x * f);
    wy = (float)(y * f);
    e += ex;
}

// One FP64 step of the slow path on the normalised delta (x, y) 2^e around the FP64
// orbit value Z: the float step's formulas with se = 2^e, the dc term (cx, cy) already
// in units of 2^e.  The result is in units of 2^e.
template <int FT>
__device__ __forceinline__ void fe32_step_fp64(const ApFrameParams& p, double Zx, double Zy, double x,
                                               double y, int e, double cx, double cy, double& nx,
                                               double& ny) {
    const double se = ldexp(1.0, e);
    if (FT == kFtQuad) {
        nx = 2.0 * (Zx * x - Zy * y) + se * (x - y) * (x + y) + cx;
        ny = 2.0 * (Zx * y + Zy * x) + se * 2.0 * x * y + cy;
    } else if (FT == kFtShip) {
        const double sx = Zx >= 0.0 ? 1.0 : -1.0, sy = Zy >= 0.0 ? 1.0 : -1.0;
        const double ddx = (Zx + x * se) * sx >= 0.0 ? sx * x : -sx * (ldexp(2.0 * Zx, -e) + x);
        const double ddy = (Zy + y * se) * sy >= 0.0 ? sy * y : -sy * (ldexp(2.0 * Zy, -e) + y);
        nx = 2.0 * (Zx * x - Zy * y) + se * (x - y) * (x + y) + cx;
        ny = 2.0 * (fabs(Zx) * ddy + fabs(Zy) * ddx + se * ddx * ddy) - cy;
    } else {
        double pr = x, pi = y, qr = Zx, qi = Zy;
        for_powers(p.gen_n, [&]() {
            const double sr = se * pr + qr, si = se * pi + qi;
            const double npr = (pr * Zx - pi * Zy) + (sr * x - si * y);
            const double npi = (pr * Zy + pi * Zx) + (sr * y + si * x);
            const double nqr = qr * Zx - qi * Zy, nqi = qr * Zy + qi * Zx;
            pr = npr;
            pi = npi;
            qr = nqr;
            qi = nqi;
        });
        nx = pr + (p.gen_kr * x - p.gen_ki * y) + cx;
        ny = pi + (p.gen_kr * y + p.gen_ki * x) + cy;
    }
}

// One FP32 step (the fast path): Z the float copy of the orbit value, (Dx, Dy) the dc
// term in units of 2^e, (kr, ki) Multibrot's k.  A Burning Ship sign test that the float
// screen cannot decide (|dz_x| >= |Z_x| / 2) reads the FP64 orbit value at orb_k.
template <int FT>
__device__ __forceinline__ void fe32_step(const ApFrameParams& p, const float4 Z, const double4* orb_k,
                                          float& wx, float& wy, int e, float S, float Dx, float Dy,
                                          float kr, float ki) {
    if (FT == kFtQuad) {
        const float tx = fmaf(Z.x, wx, -Z.y * wy);
        const float ty = fmaf(Z.x, wy, Z.y * wx);
        const float sq_x = (wx - wy) * (wx + wy);
        const float sq_y = 2.0f * wx * wy;
        const float nx = fmaf(2.0f, tx, fmaf(S, sq_x, Dx));
        const float ny = fmaf(2.0f, ty, fmaf(S, sq_y, Dy));
        wx = nx;
        wy = ny;
    } else if (FT == kFtShip) {
        const float sx = Z.x >= 0.0f ? 1.0f : -1.0f, sy = Z.y >= 0.0f ? 1.0f : -1.0f;
        float ddx = sx * wx, ddy = sy * wy;
        const bool ux = !(fabsf(wx * S) < 0.5f * fabsf(Z.x));
        const bool uy = !(fabsf(wy * S) < 0.5f * fabsf(Z.y));
        if (ux || uy) {
            const double2 Z64 = __ldg(reinterpret_cast<const double2*>(orb_k));
            const double se = ldexp(1.0, e);
            if (ux) {
                const double x = wx, s = Z64.x >= 0.0 ? 1.0 : -1.0;
                ddx = (Z64.x + x * se) * s >= 0.0 ? (float)(s * x) : (float)(-s * (ldexp(2.0 * Z64.x, -e) + x));
            }
            if (uy) {
                const double y = wy, s = Z64.y >= 0.0 ? 1.0 : -1.0;
                ddy = (Z64.y + y * se) * s >= 0.0 ? (float)(s * y) : (float)(-s * (ldexp(2.0 * Z64.y, -e) + y));
            }
        }
        const float nx = fmaf(2.0f, fmaf(Z.x, wx, -Z.y * wy), fmaf(S, (wx - wy) * (wx + wy), Dx));
        const float ny = fmaf(2.0f, fmaf(fabsf(Z.x), ddy, fmaf(fabsf(Z.y), ddx, S * (ddx * ddy))), -Dy);
        wx = nx;
        wy = ny;
    } else {
        float pr = wx, pi = wy, qr = Z.x, qi = Z.y;
        for_powers(p.gen_n, [&]() {
            const float sr = fmaf(S, pr, qr), si = fmaf(S, pi, qi);
            const float npr = fmaf(pr, Z.x, fmaf(-pi, Z.y, fmaf(sr, wx, -si * wy)));
            const float npi = fmaf(pr, Z.y, fmaf(pi, Z.x, fmaf(sr, wy, si * wx)));
            const float nqr = fmaf(qr, Z.x, -qi * Z.y), nqi = fmaf(qr, Z.y, qi * Z.x);
            pr = npr;
            pi = npi;
            qr = nqr;
            qi = nqi;
        });
        const float nx = fmaf(kr, wx, fmaf(-ki, wy, pr + Dx));
        const float ny = fmaf(kr, wy, fmaf(ki, wx, pi + Dy));
        wx = nx;
        wy = ny;
    }
}

// One FP64 direct step z <- f(z) + c of stage 2 (zx2, zy2 the squares already formed).
template <int FT>
__device__ __forceinline__ void fe32_direct_step(const ApFrameParams& p, double& zx, double& zy, double zx2,
                                                 double zy2, double cx, double cy) {
    if (FT == kFtQuad) {
        zy = 2.0 * zx * zy + cy;
        zx = zx2 - zy2 + cx;
    } else if (FT == kFtShip) {
        zy = 2.0 * fabs(zx) * fabs(zy) - cy;
        zx = zx2 - zy2 + cx;
    } else {
        double zr = zx, zi = zy;
        for_powers(p.gen_n, [&]() {
            const double nr = zr * zx - zi * zy, ni = zr * zy + zi * zx;
            zr = nr;
            zi = ni;
        });
        const double kzr = p.gen_kr * zx - p.gen_ki * zy;
        const double kzi = p.gen_kr * zy + p.gen_ki * zx;
        zx = zr + kzr + cx;
        zy = zi + kzi + cy;
    }
}

// One pixel of an FP32 coarse pass, resumable like the FP64 passes' PixelRun:
// fe32_begin sets it up, fe32_advance runs its loops -- all of them, or at most
// `budget` loop iterations (steps or leaps) per call when BUDGET is set -- and
// fe32_finish writes its outputs.  The per-frame kernel (ap_fe32.cu) runs the three
// in a row; the batch kernel (ap_batch.cu) runs fe32_advance a quantum at a time.
// Between calls the delta is kept as (wx, wy, e) exactly as the loop holds it (no
// renormalisation at a call boundary), so both give identical values.
struct Fe32Run {
    double zx, zy;    // stage 2: z itself
    double dcx, dcy;  // the pixel's offset from the reference, in units of 2^-E
    float wx, wy;     // stage 1: the delta's mantissa pair
    int e;            // stage 1: its exponent
    int idx, k, k2, m, glitch, leaps, skipped, rebases;
    int stage;        // 1 perturbation, 2 direct, 3 done
    SampleOut o;
};

// Renormalise (wx, wy) when it is not zero: max component into [1, 2), exponent to e.
__device__ __forceinline__ void fe32_normalise(float& wx, float& wy, int& e) {
    if (wx != 0.0f || wy != 0.0f) {
        const int ex = ilogb_max(wx, wy);
        if (ex != 0) {
            const float f = exp2i_f(-ex);
            wx *= f;
            wy *= f;
            e += ex;
        }
    }
}

__device__ __forceinline__ bool fe32_begin(const ApFrameParams& p, const ApFrameBuffers& b, int i, int j,
                                           Fe32Run& s) {
    s.idx = j * p.width + i;
    if (p.rebase_pass > 0 && b.glitch_in[s.idx] == 0) return false;
    // delta_c = dcm * 2^ec (normalised units: dx_hi = true spacing * 2^E).
    const double sub_offset = ((double)p.factor - 1.0) * 0.5;
    const double sub_i = (double)(i * p.factor) + sub_offset;
    const double sub_j = (double)(j * p.factor) + sub_offset;
    s.dcy = (p.ref_py - sub_j) * p.dy_hi;
    s.dcx = (sub_i - p.ref_px) * p.dx_hi;
    const bool julia = (p.fractal_type == 2 || p.fractal_type == 3);
    s.wx = julia ? (float)s.dcx : 0.0f;
    s.wy = julia ? (float)s.dcy : 0.0f;
    s.e = -p.e_scale;
    fe32_normalise(s.wx, s.wy, s.e);
    s.zx = s.zy = 0.0;
    s.k = s.m = 0;
    s.k2 = -1;
    s.glitch = s.leaps = s.skipped = s.rebases = 0;
    s.stage = 1;
    s.o = interior_sample();
    return true;
}

template <int FT, bool BLA, bool REBASE, bool BUDGET>
__device__ __forceinline__ void fe32_advance(const ApFrameParams& p, const ApFrameBuffers& b, Fe32Run& s,
                                             int budget) {
    constexpr int bias = kRadiusBias;
    const int ref_len = p.ref_len, max_iter = p.max_iter;
    const double4* __restrict__ orb = reinterpret_cast<const double4*>(b.orbit_packed);
    const float4* __restrict__ orb32 =
        reinterpret_cast<const float4*>(b.orbit_packed + 4 * (size_t)(ref_len + 1));
    const double* __restrict__ Rs = b.bla_packed;
    const Fe32Bla* __restrict__ AB =
        reinterpret_cast<const Fe32Bla*>(b.bla_packed + (size_t)ref_len * 16);
    const bool julia = (p.fractal_type == 2 || p.fractal_type == 3);
    const int ec = -p.e_scale;
    const float dcmx = (float)s.dcx, dcmy = (float)s.dcy;
    const float pdx = julia ? 0.0f : dcmx, pdy = julia ? 0.0f : dcmy;
    const float kr = (float)p.gen_kr, ki = (float)p.gen_ki;

    float wx = s.wx, wy = s.wy;
    int e = s.e;
    // The exponent-dependent scales S = 2^e, D = dcm 2^(ec - e), P2 = 2^(2e + bias).
    float S, Dx, Dy;
    double P2;
    auto refresh = [&]() {
        S = exp2i_f(e);
        const float dsc = exp2i_f(ec - e);
        Dx = pdx * dsc;
        Dy = pdy * dsc;
        P2 = exp2i_d(2 * e + bias);
    };
    auto rescale = [&]() {
        fe32_normalise(wx, wy, e);
        refresh();
    };
    refresh();

    const bool strict = !REBASE && p.strict_glitch > 0;
    // k: the reference index (and, without rebasing, the pixel's iterations).  With
    // rebasing the pixel's iterations are k + (max_iter - lim): a restart moves lim.
    int k = REBASE ? s.m : s.k;
    int lim = REBASE ? max_iter - s.k + s.m : max_iter;
    int glitch = s.glitch, leaps = s.leaps, skipped = s.skipped, k2 = s.k2, rebases = s.rebases;
    const int max_level = p.bla_levels - 1;
    SampleOut o = s.o;
    bool finished = false, paused = false;
    const double inv_ln = inv_ln_for(p.fractal_type, p.gen_n);

    while (s.stage == 1 && (REBASE ? (k < lim) : (k < ref_len))) {
        if (BUDGET && --budget < 0) {
            paused = true;
            break;
        }
        const float4 Z = __ldg(orb32 + k);
        const float wm2 = wx * wx + wy * wy;
        if (REBASE) {
            // z is formed in FP64 where a test can fire: at the end of the reference, at a
            // close approach, near escape, or where |dz| > |Z| / 2 (|Z + dz| < |dz| needs it)
            bool test = k == ref_len || Z.w != 0.0f || (e >= -53 && wm2 * (S * S) > 0.2f * Z.z);
            if (!test && e >= -40) {
                const float zx = Z.x + wx * S, zy = Z.y + wy * S;
                test = zx * zx + zy * zy > 65535.0f;
            }
            if (test) {
                const double2 Z64 = __ldg(reinterpret_cast<const double2*>(orb + k));
                const double sc = ldexp(1.0, e), x = wx, y = wy;
                const double ax = Z64.x + x * sc, ay = Z64.y + y * sc;
                const double mag2 = ax * ax + ay * ay;
                if (!(mag2 <= kBailout)) {
                    const int kk = k + (max_iter - lim);
                    if (isnan(mag2)) {
                        o.s = (float)kk;
                        o.s64 = (double)kk;
                        o.k = kk;
                        glitch = 1;
                    } else {
                        o = escaped_sample(kk, mag2, inv_ln);
                    }
                    finished = true;
                    break;
                }
                // |z| < |dz| compared in units of 2^e, so that neither side underflows
                double bx = ldexp(Z64.x, -e) + x, by = ldexp(Z64.y, -e) + y;
                if ((k == ref_len && k > 0) || bx * bx + by * by < x * x + y * y) {
                    if (!(fabs(bx) + fabs(by) < 1e300)) {  // a reference that ended far above the delta
                        bx = ax;
                        by = ay;
                        e = 0;
                    }
                    renorm_to_float(bx, by, wx, wy, e);
                    rescale();
                    lim -= k;
                    k = 0;
                    ++rebases;
                    continue;
                }
            }
        } else if (e >= -40 || (strict && k > 15 && e >= -75)) {
            // Escape and Pauldelbrot tests can only fire once the delta is not negligible.
            const float zx = Z.x + wx * S, zy = Z.y + wy * S;
            const float zm2 = zx * zx + zy * zy;
            const bool near_escape = e >= -40 && zm2 > 65535.0f;
            const bool near_glitch = strict && k > 15 && zm2 < 2e-6f * Z.z;
            if (near_escape || near_glitch) {
                const double2 Z64 = __ldg(reinterpret_cast<const double2*>(orb + k));
                const double sc = ldexp(1.0, e);
                const double ax = Z64.x + (double)wx * sc, ay = Z64.y + (double)wy * sc;
                const double mag2 = ax * ax + ay * ay;
                if (mag2 > kBailout) {
                    o = escaped_sample(k, mag2, inv_ln);
                    finished = true;
                    break;
                }
                if (near_glitch) {
                    const double r2 = Z64.x * Z64.x + Z64.y * Z64.y;
                    const double thr = r2 > 1e-8 ? 1e-6 * r2 : -1.0;  // as the reference forms it
                    if (mag2 < thr) glitch = 1;
                }
            }
        }
        if (BLA && k < ref_len - 1) {
            const double dzs = (double)wm2 * P2;
            const double* row = Rs + (size_t)k * 16;
            if (dzs < __ldg(row)) {
                int lo = 0, hi = max_level;
                if (REBASE) hi = min(hi, 31 - __clz(lim - k));  // the leap ends at or before max_iter
#pragma unroll 4
                for (int it = 0; it < 4; ++it) {
                    if (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (dzs < __ldg(row + mid)) lo = mid;
                        else hi = mid - 1;
                    }
                }
                const Fe32Bla c = AB[(size_t)k * 16 + lo];
                // dz' = A dz + B dc = 2^(e + ea) [am w + bm dcm 2^(eb + ec - e - ea)]
                const int fe = c.eb + ec - e - c.ea;
                if (fe >= -120 && fe <= 120) {
                    const float f = exp2i_f(fe);
                    const float bx = (c.br * pdx - c.bi * pdy) * f;
                    const float by = (c.br * pdy + c.bi * pdx) * f;
                    const float nx = fmaf(c.ar, wx, fmaf(-c.ai, wy, bx));
                    const float ny = fmaf(c.ar, wy, fmaf(c.ai, wx, by));
                    wx = nx;
                    wy = ny;
                    e += c.ea;
                } else {  // FP64 slow path: the dc term's scale leaves the float range
                    const double bx = ldexp((double)c.br * pdx - (double)c.bi * pdy, fe);
                    const double by = ldexp((double)c.br * pdy + (double)c.bi * pdx, fe);
                    const double nx = (double)c.ar * wx - (double)c.ai * wy + bx;
                    const double ny = (double)c.ar * wy + (double)c.ai * wx + by;
                    e += c.ea;
                    renorm_to_float(nx, ny, wx, wy, e);
                }
                rescale();
                k += 1 << lo;
                ++leaps;
                skipped += 1 << lo;
                continue;
            }
        }
        if (Z.w != 0.0f || ec - e > 120) {
            // FP64 slow path: the same step on the FP64 orbit, dc term dcm 2^(ec - e).
            const double2 Z64 = __ldg(reinterpret_cast<const double2*>(orb + k));
            double nx, ny;
            fe32_step_fp64<FT>(p, Z64.x, Z64.y, wx, wy, e, ldexp((double)pdx, ec - e),
                               ldexp((double)pdy, ec - e), nx, ny);
            renorm_to_float(nx, ny, wx, wy, e);
            rescale();
            ++k;
            continue;
        }
        fe32_step<FT>(p, Z, orb + k, wx, wy, e, S, Dx, Dy, kr, ki);
        const float mx = fmaxf(fabsf(wx), fabsf(wy));
        if (mx > 65536.0f || (mx < 1.52587890625e-05f && mx > 0.0f)) rescale();
        ++k;
    }
    s.wx = wx;
    s.wy = wy;
    s.e = e;
    s.glitch = glitch;
    s.leaps = leaps;
    s.skipped = skipped;
    s.rebases = rebases;
    if (REBASE) {
        s.m = k;
        s.k = k + (max_iter - lim);
        if (!paused) {
            s.stage = 3;
            if (finished) s.k = o.k;
        }
        s.o = o;
        return;
    }
    if (paused || finished) {
        s.k = k;
        if (finished) s.stage = 3;
        s.o = o;
        return;
    }
    // Stage 2: FP64 direct iteration from Z_ref_len + dz, c = ref_c + dc.
    const double dct_x = s.dcx * ldexp(1.0, ec), dct_y = s.dcy * ldexp(1.0, ec);
    const double cx = julia ? p.julia_cx_hi : p.ref_cx + dct_x;
    const double cy = julia ? p.julia_cy_hi : p.ref_cy + dct_y;
    double zx = s.zx, zy = s.zy;
    if (s.stage == 1) {
        const double2 Zend = __ldg(reinterpret_cast<const double2*>(orb + ref_len));
        const double sc = ldexp(1.0, e);
        zx = Zend.x + (double)wx * sc;
        zy = Zend.y + (double)wy * sc;
        // a pixel that escapes together with the reference (at k = ref_len) is not glitched
        if (!(zx * zx + zy * zy > kBailout) && ref_len < max_iter) glitch = 1;
        k2 = k;
        s.stage = 2;
    }
    const bool nan_guard = (p.flags & AP_FLAG_NAN_GUARD) != 0;
    while (k < max_iter) {
        if (BUDGET && --budget < 0) {
            paused = true;
            break;
        }
        const double zx2 = zx * zx, zy2 = zy * zy;
        const double mag2 = zx2 + zy2;
        if (nan_guard && (isnan(mag2) || isinf(mag2))) {
            o.s = (float)k;
            o.s64 = (double)k;
            o.k = k;
            glitch = 1;
            break;
        }
        if (mag2 > kBailout) {
            o = escaped_sample(k, mag2, inv_ln);
            break;
        }
        fe32_direct_step<FT>(p, zx, zy, zx2, zy2, cx, cy);
        ++k;
    }
    s.zx = zx;
    s.zy = zy;
    s.k = k;
    s.k2 = k2;
    s.glitch = glitch;
    s.o = o;
    if (!paused) s.stage = 3;
}

__device__ __forceinline__ void fe32_finish(const ApFrameParams& p, const ApFrameBuffers& b, const Fe32Run& s) {
    const int k_end = (s.o.k == -1) ? p.max_iter : s.k;
    b.iter_map[s.idx] = s.o.s;
    if (b.kmap) b.kmap[s.idx] = s.o.k;
    if (b.s64) b.s64[s.idx] = s.o.s64;
    if (b.glitch_out) b.glitch_out[s.idx] = s.glitch ? 1 : 0;
    if (b.counters) {
        const int it1 = (s.k2 < 0 ? k_end : s.k2) - s.skipped;
        const int it2 = s.k2 < 0 ? 0 : k_end - s.k2;
        reinterpret_cast<int4*>(b.counters)[s.idx] = make_int4(it1, s.leaps, it2, s.rebases);
    }
}

}  // namespace ap
