// ap_coarse.cuh -- one pixel of a coarse FP64-delta perturbation pass on packed inputs.
//
// Same results as the generic render pass (ap_perturb.cuh) for tier
// AP_TIER_PERTURB in AP_MODE_COARSE without in-kernel colouring; it is picked
// by ap_render_pass when the buffers carry the packed orbit (ap_pack_orbit)
// and, with BLA, the packed table (ap_pack_bla).  What changes is only how the
// loop gets its inputs:
//   * one 32-byte read per step: Z_k, a safe radius and the level-0 BLA
//     radius.  While |dz| is below the safe radius neither the escape test nor
//     the Pauldelbrot test can fire, so |Z + dz|^2 and the threshold are not
//     formed (the rounded |dz|^2 decides, and the BLA test reuses it);
//   * the 16 BLA radii of step k in one 128-byte row.  Radii never increase
//     with the level (each level's radius is the min of its first half's), and
//     levels past the end of the orbit hold 0, so the largest admissible level
//     -- the reference's top-down scan -- is found by a 4-probe binary search;
//   * formula, BLA presence and arithmetic profile are template parameters;
//   * no colouring (ap_colour runs afterwards), keeping registers low.
#pragma once

#include "ap_common.cuh"

#ifndef AP_REBASE_PREFETCH
#define AP_REBASE_PREFETCH 0
#endif

namespace ap {

constexpr int kFtQuad = 0;   // Mandelbrot (0) and its Julia set (2)
constexpr int kFtShip = 1;   // Burning Ship (1) and its Julia set (3)
constexpr int kFtMulti = 4;  // Multibrot z^n + k z + c

// Calls power() n - 1 times, the common degrees unrolled: the same operations in the
// same order, and what the last call prepares for a next one is dead and goes.
template <typename F>
__device__ __forceinline__ void for_powers(int n, F&& power) {
    switch (n) {
    case 2: power(); break;
    case 3: power(); power(); break;
    case 4: power(); power(); power(); break;
    case 5: power(); power(); power(); power(); break;
    default:
        for (int t = 0; t < n - 1; ++t) power();
    }
}

// 32-byte record through the read-only path (two 16-byte loads).
__device__ __forceinline__ double4 ldg4(const double4* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    const double2 a = __ldg(q), c = __ldg(q + 1);
    return make_double4(a.x, a.y, c.x, c.y);
}

// One pixel of a coarse pass, resumable: pixel_begin sets it up, pixel_advance runs
// its stage-1 (perturbation) and stage-2 (direct) loops -- all of them, or at most
// `budget` loop iterations (steps or leaps) per call when BUDGET is set, so that a
// persistent kernel can hand a lane whose pixel finished a new one -- and
// pixel_finish writes its outputs.  coarse_pixel runs the three in a row; the
// per-frame kernel below and the batch kernel (ap_batch.cu) share this code, so both
// give identical values.
struct PixelRun {
    double dzx, dzy;  // stage 1: the delta
    double zx, zy;    // stage 2: z itself
    double dcx, dcy;  // the pixel's offset from the reference
    int idx, k, k0, k2, glitch, leaps, skipped;
    int stage;        // 1 perturbation, 2 direct, 3 done
    int m, rebases;   // one-pass rebasing: reference index (k counts iterations), restarts
    SampleOut o;
};

template <int ARITH, int FT>
__device__ __forceinline__ bool pixel_begin(const ApFrameParams& p, const ApFrameBuffers& b, int i, int j,
                                            PixelRun& s) {
    s.idx = j * p.width + i;
    if (p.rebase_pass > 0 && b.glitch_in[s.idx] == 0) return false;
    const double sub_offset = ((double)p.factor - 1.0) * 0.5;
    const double sub_i = (double)(i * p.factor) + sub_offset;
    const double sub_j = (double)(j * p.factor) + sub_offset;
    s.dcy = (p.ref_py - sub_j) * p.dy_hi;
    s.dcx = (sub_i - p.ref_px) * p.dx_hi;
    const bool julia = (p.fractal_type == 2 || p.fractal_type == 3);
    s.dzx = julia ? s.dcx : 0.0;
    s.dzy = julia ? s.dcy : 0.0;
    s.k = 0;
    if (p.bbsa_skip > 0 && FT != kFtShip) {
        const double ux = s.dcx * p.bbsa_inv_r, uy = s.dcy * p.bbsa_inv_r;
        if (ux * ux + uy * uy <= 1.0) {
            bool eight = false;
            for (int q = 8; q < 16; ++q) eight |= (p.bbsa[q] != 0.0);
            const int top = eight ? 7 : 3;
            double tr = ux * p.bbsa[2 * top] - uy * p.bbsa[2 * top + 1];
            double ti = ux * p.bbsa[2 * top + 1] + uy * p.bbsa[2 * top];
            for (int q = top - 1; q >= 0; --q) {
                const double ar = p.bbsa[2 * q] + tr, ai = p.bbsa[2 * q + 1] + ti;
                tr = ux * ar - uy * ai;
                ti = ux * ai + uy * ar;
            }
            s.dzx = tr;
            s.dzy = ti;
            s.k = p.bbsa_skip;
        }
    }
    s.k0 = s.k;
    s.m = s.k;
    s.rebases = 0;
    s.k2 = -1;
    s.glitch = s.leaps = s.skipped = 0;
    s.stage = 1;
    s.o = interior_sample();
    return true;
}

template <int ARITH, int FT, bool BLA, bool BUDGET>
__device__ __forceinline__ void pixel_advance(const ApFrameParams& p, const ApFrameBuffers& b, PixelRun& s,
                                              int budget) {
    constexpr bool kCpu = (ARITH == AP_ARITH_REF_CPU);
    const bool julia = (p.fractal_type == 2 || p.fractal_type == 3);
    const int ref_len = p.ref_len, max_iter = p.max_iter;
    const double4* __restrict__ orb = reinterpret_cast<const double4*>(b.orbit_packed);
    const double inv_ln = inv_ln_for(p.fractal_type, p.gen_n);
    int k = s.k, glitch = s.glitch, leaps = s.leaps, skipped = s.skipped;
    SampleOut o = s.o;

    if (s.stage == 1) {
        double dzx = s.dzx, dzy = s.dzy;
        const double dcpx = julia ? 0.0 : s.dcx, dcpy = julia ? 0.0 : s.dcy;
        const bool strict = p.strict_glitch > 0;
        const bool esc_glitch = (p.flags & AP_FLAG_ESCAPE_GLITCH) != 0;
        const double* __restrict__ R = b.bla_packed;
        const double4* __restrict__ AB =
            reinterpret_cast<const double4*>(b.bla_packed + (size_t)ref_len * 16);
        const int max_level = p.bla_levels - 1;
        bool finished = false, paused = false;
        while (k < ref_len) {
            if (BUDGET && --budget < 0) {
                paused = true;
                break;
            }
            const double4 Z = ldg4(orb + k);
            const double rx = Z.x, ry = Z.y;
            const double zx = rx + dzx, zy = ry + dzy;
            const double dz_mag2 = dzx * dzx + dzy * dzy;
            // One branch on the common path: inside the safe radius (no test can fire)
            // and outside the level-0 BLA radius (no leap), the step runs straight
            // through.  The packed radii are 0 wherever k + 2^d >= ref_len, so no level
            // is admissible at the last step without a separate bound check.
            const bool unsafe = !(dz_mag2 < Z.z);
            const bool leap = BLA && (dz_mag2 < Z.w);
            if (unsafe || leap) {
                if (unsafe) {
                    const double mag2 = zx * zx + zy * zy;
                    const double r_mag2 = rx * rx + ry * ry;
                    if (mag2 > kBailout) {
                        if (esc_glitch && strict && k > 15 && r_mag2 < 4.0) glitch = 1;
                        o = escaped_sample(k, mag2, inv_ln);
                        finished = true;
                        break;
                    }
                    // the Pauldelbrot threshold, as the reference forms it
                    const double thr = r_mag2 > 1e-8 ? 1e-6 * r_mag2 : -1.0;
                    if (strict && k > 15 && mag2 < thr) glitch = 1;
                }
                if (leap) {
                    const double* row = R + (size_t)k * 16;
                    int hi = max_level;
                    if (dz_mag2 == 0.0 && (dzx != 0.0 || dzy != 0.0)) hi = min(hi, 8);
                    // The admissible levels are a prefix 0..lo (radii never increase
                    // with the level), so lo is a count.  Two rounds of three
                    // independent loads: the quarter of the row, then the level in it.
                    int q = 0;
#pragma unroll
                    for (int t = 1; t <= 3; ++t)
                        q += (4 * t <= hi && dz_mag2 < __ldg(row + 4 * t)) ? 1 : 0;
                    int lo = 4 * q;
#pragma unroll
                    for (int t = 1; t <= 3; ++t) {
                        const int d = 4 * q + t;
                        lo += (d <= hi && dz_mag2 < __ldg(row + d)) ? 1 : 0;
                    }
                    const double4 e = ldg4(AB + (size_t)k * 16 + lo);
                    double nx, ny;
                    if (kCpu) {
                        nx = (e.x * dzx - e.y * dzy) + (e.z * dcpx - e.w * dcpy);
                        ny = (e.x * dzy + e.y * dzx) + (e.z * dcpy + e.w * dcpx);
                    } else {
                        nx = fma(e.x, dzx, fma(-e.y, dzy, fma(e.z, dcpx, -e.w * dcpy)));
                        ny = fma(e.x, dzy, fma(e.y, dzx, fma(e.z, dcpy, e.w * dcpx)));
                    }
                    dzx = nx;
                    dzy = ny;
                    if (isnan(dzx) || isnan(dzy) || isinf(dzx) || isinf(dzy)) {
                        o = interior_sample();
                        o.s = (float)k;
                        o.s64 = (double)k;
                        o.k = k;
                        glitch = 1;
                        finished = true;
                        break;
                    }
                    k += 1 << lo;
                    ++leaps;
                    skipped += 1 << lo;
                    continue;
                }
            }
            if (FT == kFtQuad) {
                double nx, ny;
                if (kCpu) {
                    nx = (2.0 * rx + dzx) * dzx - (2.0 * ry + dzy) * dzy + dcpx;
                    ny = 2.0 * (zx * dzy + ry * dzx) + dcpy;
                } else {
                    nx = fma(2.0 * rx + dzx, dzx, fma(-(2.0 * ry + dzy), dzy, dcpx));
                    ny = fma(2.0, fma(zx, dzy, ry * dzx), dcpy);
                }
                dzx = nx;
                dzy = ny;
            } else if (FT == kFtShip) {
                const double nx = (2.0 * rx + dzx) * dzx - (2.0 * ry + dzy) * dzy + dcpx;
                const double sx = rx >= 0.0 ? 1.0 : -1.0, sy = ry >= 0.0 ? 1.0 : -1.0;
                const double ddx = zx * sx >= 0.0 ? sx * dzx : -sx * (2.0 * rx + dzx);
                const double ddy = zy * sy >= 0.0 ? sy * dzy : -sy * (2.0 * ry + dzy);
                dzy = 2.0 * (fabs(rx) * ddy + fabs(ry) * ddx + ddx * ddy) - dcpy;
                dzx = nx;
            } else {
                double pr = dzx, pi = dzy, qr = rx, qi = ry;
                for_powers(p.gen_n, [&]() {
                    const double t1r = pr * rx - pi * ry, t1i = pr * ry + pi * rx;
                    const double sr = pr + qr, si = pi + qi;
                    const double t2r = sr * dzx - si * dzy, t2i = sr * dzy + si * dzx;
                    pr = t1r + t2r;
                    pi = t1i + t2i;
                    const double nqr = qr * rx - qi * ry, nqi = qr * ry + qi * rx;
                    qr = nqr;
                    qi = nqi;
                });
                const double kzr = p.gen_kr * dzx - p.gen_ki * dzy;
                const double kzi = p.gen_kr * dzy + p.gen_ki * dzx;
                dzx = pr + kzr + dcpx;
                dzy = pi + kzi + dcpy;
            }
            ++k;
        }
        if (paused) {
            s.dzx = dzx;
            s.dzy = dzy;
            s.k = k;
            s.glitch = glitch;
            s.leaps = leaps;
            s.skipped = skipped;
            return;
        }
        if (finished) {
            s.stage = 3;
        } else {
            // Stage 2: past the end of the reference orbit, iterate z directly.
            const double4 Zend = ldg4(orb + ref_len);
            s.zx = Zend.x + dzx;
            s.zy = Zend.y + dzy;
            if (ref_len < max_iter) glitch = 1;
            s.k2 = k;
            o = interior_sample();
            s.stage = 2;
        }
    }

    if (s.stage == 2) {
        double zx = s.zx, zy = s.zy;
        const double cx = julia ? p.julia_cx_hi : p.ref_cx + s.dcx;
        const double cy = julia ? p.julia_cy_hi : p.ref_cy + s.dcy;
        const bool nan_guard = (p.flags & AP_FLAG_NAN_GUARD) != 0;
        bool paused = false;
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
            ++k;
        }
        s.zx = zx;
        s.zy = zy;
        if (!paused) s.stage = 3;
    }
    s.k = k;
    s.glitch = glitch;
    s.leaps = leaps;
    s.skipped = skipped;
    s.o = o;
}

// One-pass rebasing (AP_FLAG_REBASE), for orbits that start at Z_0 = 0 (fractal
// types 0, 1, 4).  k counts the pixel's iterations, m indexes the reference.  At
// each step z = Z_m + dz is tested for escape; when |z| < |dz| -- the delta has
// outgrown the value it perturbs, where a plain delta would lose its precision --
// or when the reference has ended (m == ref_len), the delta restarts from the start
// of the orbit: dz <- z, m <- 0 (Zhuoran, fractalforums.org 2021).  A pixel is never
// flagged glitched (only a NaN/Inf delta is) and never falls back to direct
// iteration, so one pass serves every pixel.  The packed safe radius also rules
// out the rebase test (|dz| < |Z|/2), so the common path is the same single branch
// as pixel_advance's.  Leaps are capped so that k never passes max_iter.  ARITH may
// also be AP_ARITH_FAST: |dz|^2, |z|^2 and every formula's step as fused multiply-adds
// (about 10 FP64 instructions per Mandelbrot step on the common path; a Multibrot
// power costs 14 instead of 22), leaps as the CUDA profile.
template <int ARITH, int FT, bool BLA, bool BUDGET>
__device__ __forceinline__ void rebase_advance(const ApFrameParams& p, const ApFrameBuffers& b, PixelRun& s,
                                               int budget) {
    constexpr bool kCpu = (ARITH == AP_ARITH_REF_CPU);
    constexpr bool kFast = (ARITH == AP_ARITH_FAST);
    const int ref_len = p.ref_len, max_iter = p.max_iter;
    const double4* __restrict__ orb = reinterpret_cast<const double4*>(b.orbit_packed);
    const double inv_ln = inv_ln_for(p.fractal_type, p.gen_n);
    const double* __restrict__ R = b.bla_packed;
    const double4* __restrict__ AB = reinterpret_cast<const double4*>(b.bla_packed + (size_t)ref_len * 16);
    const int max_level = p.bla_levels - 1;
    const double dcpx = s.dcx, dcpy = s.dcy;
    // k (the pixel's iterations) is not kept: a step or a leap moves k and m alike and a
    // restart moves only m, so k = m + (max_iter - lim) with lim moved at each restart,
    // and the loop runs while m < lim (k < max_iter).
    int m = s.m, lim = max_iter - s.k + s.m;
    int glitch = s.glitch, leaps = s.leaps, skipped = s.skipped, rebases = s.rebases;
    double dzx = s.dzx, dzy = s.dzy;
    SampleOut o = s.o;
    bool paused = false;
#if AP_REBASE_PREFETCH
    double4 Znext = ldg4(orb + m);
#endif
    while (m < lim) {
        if (BUDGET && --budget < 0) {
            paused = true;
            break;
        }
#if AP_REBASE_PREFETCH
        // the record of the common path's next step is requested one step ahead
        const double4 Z = Znext;
        Znext = ldg4(orb + min(m + 1, ref_len));
#else
        const double4 Z = ldg4(orb + m);
#endif
        const double rx = Z.x, ry = Z.y;
        // z itself: every step but the fused Mandelbrot one uses it; that one forms it
        // only where a test can fire
        constexpr bool kLateZ = kFast && FT == kFtQuad;
        double zx = 0.0, zy = 0.0;
        if (!kLateZ) {
            zx = rx + dzx;
            zy = ry + dzy;
        }
        const double dz_mag2 = kFast ? fma(dzx, dzx, dzy * dzy) : dzx * dzx + dzy * dzy;
        // ap_pack_orbit leaves the orbit's last record (m == ref_len) with safe radius 0,
        // so the end of the reference takes this branch without a test of its own
        const bool unsafe = !(dz_mag2 < Z.z);
        const bool leap = BLA && (dz_mag2 < Z.w);
        if (unsafe || leap) {
            if (unsafe) {
                if (kLateZ) {
                    zx = rx + dzx;
                    zy = ry + dzy;
                }
                const double mag2 = kFast ? fma(zx, zx, zy * zy) : zx * zx + zy * zy;
                if (!(mag2 <= kBailout)) {
                    const int k = m + (max_iter - lim);
                    if (isnan(mag2)) {
                        o = interior_sample();
                        o.s = (float)k;
                        o.s64 = (double)k;
                        o.k = k;
                        glitch = 1;
                    } else {
                        o = escaped_sample(k, mag2, inv_ln);
                    }
                    s.stage = 3;
                    break;
                }
                if (mag2 < dz_mag2 || (m == ref_len && m > 0)) {
                    dzx = zx;
                    dzy = zy;
                    lim -= m;
                    m = 0;
                    ++rebases;
#if AP_REBASE_PREFETCH
                    Znext = ldg4(orb);
#endif
                    continue;
                }
            }
            if (leap) {
                const double* row = R + (size_t)m * 16;
                int hi = max_level;
                if (dz_mag2 == 0.0 && (dzx != 0.0 || dzy != 0.0)) hi = min(hi, 8);
                hi = min(hi, 31 - __clz(lim - m));  // k + 2^lo <= max_iter
                int q = 0;
#pragma unroll
                for (int t = 1; t <= 3; ++t)
                    q += (4 * t <= hi && dz_mag2 < __ldg(row + 4 * t)) ? 1 : 0;
                int lo = 4 * q;
#pragma unroll
                for (int t = 1; t <= 3; ++t) {
                    const int d = 4 * q + t;
                    lo += (d <= hi && dz_mag2 < __ldg(row + d)) ? 1 : 0;
                }
                const double4 e = ldg4(AB + (size_t)m * 16 + lo);
                double nx, ny;
                if (kCpu) {
                    nx = (e.x * dzx - e.y * dzy) + (e.z * dcpx - e.w * dcpy);
                    ny = (e.x * dzy + e.y * dzx) + (e.z * dcpy + e.w * dcpx);
                } else {
                    nx = fma(e.x, dzx, fma(-e.y, dzy, fma(e.z, dcpx, -e.w * dcpy)));
                    ny = fma(e.x, dzy, fma(e.y, dzx, fma(e.z, dcpy, e.w * dcpx)));
                }
                dzx = nx;
                dzy = ny;
                if (isnan(dzx) || isnan(dzy) || isinf(dzx) || isinf(dzy)) {
                    const int k = m + (max_iter - lim);
                    o = interior_sample();
                    o.s = (float)k;
                    o.s64 = (double)k;
                    o.k = k;
                    glitch = 1;
                    s.stage = 3;
                    break;
                }
                m += 1 << lo;
                ++leaps;
                skipped += 1 << lo;
#if AP_REBASE_PREFETCH
                Znext = ldg4(orb + m);
#endif
                continue;
            }
        }
        if (FT == kFtQuad) {
            double nx, ny;
            if (kFast) {  // (2Z + dz) dz + dc with a = 2Z + dz rounded once
                const double ax = fma(2.0, rx, dzx), ay = fma(2.0, ry, dzy);
                nx = fma(ax, dzx, fma(-ay, dzy, dcpx));
                ny = fma(ax, dzy, fma(ay, dzx, dcpy));
            } else if (kCpu) {
                nx = (2.0 * rx + dzx) * dzx - (2.0 * ry + dzy) * dzy + dcpx;
                ny = 2.0 * (zx * dzy + ry * dzx) + dcpy;
            } else {
                nx = fma(2.0 * rx + dzx, dzx, fma(-(2.0 * ry + dzy), dzy, dcpx));
                ny = fma(2.0, fma(zx, dzy, ry * dzx), dcpy);
            }
            dzx = nx;
            dzy = ny;
        } else if (FT == kFtShip) {
            const double sx = rx >= 0.0 ? 1.0 : -1.0, sy = ry >= 0.0 ? 1.0 : -1.0;
            if (kFast) {  // 2Z + dz rounded once (2Z is exact); products fused into the sums
                const double ax = fma(2.0, rx, dzx), ay = fma(2.0, ry, dzy);
                const double nx = fma(ax, dzx, fma(-ay, dzy, dcpx));
                const double ddx = zx * sx >= 0.0 ? sx * dzx : -sx * ax;
                const double ddy = zy * sy >= 0.0 ? sy * dzy : -sy * ay;
                dzy = fma(2.0, fma(fabs(rx), ddy, fma(fabs(ry), ddx, ddx * ddy)), -dcpy);
                dzx = nx;
            } else {
                const double nx = (2.0 * rx + dzx) * dzx - (2.0 * ry + dzy) * dzy + dcpx;
                const double ddx = zx * sx >= 0.0 ? sx * dzx : -sx * (2.0 * rx + dzx);
                const double ddy = zy * sy >= 0.0 ? sy * dzy : -sy * (2.0 * ry + dzy);
                dzy = 2.0 * (fabs(rx) * ddy + fabs(ry) * ddx + ddx * ddy) - dcpy;
                dzx = nx;
            }
        } else if (kFast) {
            // (Z + dz)^n - Z^n by P_{j+1} = P_j Z + (P_j + Z^j) dz, each complex product
            // sum as one chain of fused multiply-adds, then + k dz + dc
            double pr = dzx, pi = dzy, qr = rx, qi = ry;
            for_powers(p.gen_n, [&]() {
                const double sr = pr + qr, si = pi + qi;
                const double npr = fma(pr, rx, fma(-pi, ry, fma(sr, dzx, -si * dzy)));
                const double npi = fma(pr, ry, fma(pi, rx, fma(sr, dzy, si * dzx)));
                const double nqr = fma(qr, rx, -qi * ry), nqi = fma(qr, ry, qi * rx);
                pr = npr;
                pi = npi;
                qr = nqr;
                qi = nqi;
            });
            const double ox = dzx, oy = dzy;
            dzx = fma(p.gen_kr, ox, fma(-p.gen_ki, oy, pr + dcpx));
            dzy = fma(p.gen_kr, oy, fma(p.gen_ki, ox, pi + dcpy));
        } else {
            double pr = dzx, pi = dzy, qr = rx, qi = ry;
            for_powers(p.gen_n, [&]() {
                const double t1r = pr * rx - pi * ry, t1i = pr * ry + pi * rx;
                const double sr = pr + qr, si = pi + qi;
                const double t2r = sr * dzx - si * dzy, t2i = sr * dzy + si * dzx;
                pr = t1r + t2r;
                pi = t1i + t2i;
                const double nqr = qr * rx - qi * ry, nqi = qr * ry + qi * rx;
                qr = nqr;
                qi = nqi;
            });
            const double kzr = p.gen_kr * dzx - p.gen_ki * dzy;
            const double kzi = p.gen_kr * dzy + p.gen_ki * dzx;
            dzx = pr + kzr + dcpx;
            dzy = pi + kzi + dcpy;
        }
        ++m;
    }
    if (!paused) s.stage = 3;
    s.dzx = dzx;
    s.dzy = dzy;
    s.k = m + (max_iter - lim);
    s.m = m;
    s.glitch = glitch;
    s.leaps = leaps;
    s.skipped = skipped;
    s.rebases = rebases;
    s.o = o;
}

__device__ __forceinline__ void pixel_finish(const ApFrameParams& p, const ApFrameBuffers& b, const PixelRun& s) {
    const int max_iter = p.max_iter;
    const int k_end = (s.o.k == -1) ? max_iter : s.k;
    b.iter_map[s.idx] = s.o.s;
    if (b.kmap) b.kmap[s.idx] = s.o.k;
    if (b.s64) b.s64[s.idx] = s.o.s64;
    if (b.glitch_out) b.glitch_out[s.idx] = s.glitch ? 1 : 0;
    if (b.counters) {
        const int it1 = (s.k2 < 0 ? k_end - s.k0 : s.k2 - s.k0) - s.skipped;
        const int it2 = s.k2 < 0 ? 0 : k_end - s.k2;
        reinterpret_cast<int4*>(b.counters)[s.idx] = make_int4(it1, s.leaps, it2, s.rebases);
    }
}

// One pixel (i, j) of a coarse pass, start to finish (REBASE: AP_FLAG_REBASE).
template <int ARITH, int FT, bool BLA, bool REBASE>
__device__ __forceinline__ void coarse_pixel(const ApFrameParams& p, const ApFrameBuffers& b, int i,
                                             int j) {
    PixelRun s;
    if (!pixel_begin<ARITH, FT>(p, b, i, j, s)) return;
    if (REBASE)
        rebase_advance<ARITH, FT, BLA, false>(p, b, s, 0);
    else
        pixel_advance<ARITH, FT, BLA, false>(p, b, s, 0);
    pixel_finish(p, b, s);
}

}  // namespace ap
