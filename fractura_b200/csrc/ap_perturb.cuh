// ap_perturb.cuh -- perturbation tiers.
//
// FP64 deltas: delta_{k+1} = 2 Z_k delta_k + delta_k^2 + delta_c around a
// host-computed reference orbit Z (read from HBM/L2 through the read-only
// path), with chained-BLA leaps delta <- A delta + B delta_c taken from the
// largest table level whose validity radius covers |delta|.
//
// Semantics of cpu_compute_perturbation_sample (math_core/cpu_kernels.py:374-602)
// and of the CUDA variants compute_perturbation_sample /
// compute_perturbation_sample_bla (math_core/cuda_kernels.py:422-815); the
// variant differences are the AP_FLAG_ESCAPE_GLITCH / AP_FLAG_NAN_GUARD flags,
// the arithmetic differences are ARITH.
#pragma once

#include "ap_common.cuh"

namespace ap {

struct cplx {
    double r, i;
};

__device__ __forceinline__ cplx cmul(double ar, double ai, double br, double bi) {
    return {ar * br - ai * bi, ar * bi + ai * br};
}

// Series-approximation start (math_core/cpu_kernels.py:206-223), u = delta_c / r.
__device__ __forceinline__ cplx bbsa_eval(const double* c, double ux, double uy) {
    bool eight = false;
#pragma unroll
    for (int q = 8; q < 16; ++q) eight |= (c[q] != 0.0);
    const int top = eight ? 7 : 3;
    cplx t = cmul(ux, uy, c[2 * top], c[2 * top + 1]);
    for (int q = top - 1; q >= 0; --q) t = cmul(ux, uy, c[2 * q] + t.r, c[2 * q + 1] + t.i);
    return t;
}

__device__ __forceinline__ SampleOut glitch_sample(int k) {
    SampleOut o = interior_sample();
    o.s = (float)k;
    o.s64 = (double)k;
    o.k = k;
    o.glitch = 1;
    return o;
}

// One-pass rebasing (AP_FLAG_REBASE; fractal types 0, 1, 4, whose orbits start at
// Z_0 = 0): k counts the pixel's iterations, m indexes the reference.  z = Z_m + dz
// is tested for escape at every step; when |z| < |dz| or the reference has ended
// (m == ref_len) the delta restarts from the orbit's start, dz <- z, m <- 0
// (Zhuoran, fractalforums.org 2021).  The leap takes the largest admissible level
// that ends before the orbit does and does not carry k past max_iter.  Same values as
// the packed coarse kernel's rebase_advance (ap_coarse.cuh), AP_ARITH_FAST included.
template <int ARITH>
__device__ __forceinline__ SampleOut rebase_sample_at(const ApFrameParams& p, const ApFrameBuffers& b,
                                                      double sub_i, double sub_j) {
    constexpr bool kCpu = (ARITH == AP_ARITH_REF_CPU);
    const bool fast = !kCpu && p.arith == AP_ARITH_FAST;  // served by the CUDA-profile instance
    const int ft = p.fractal_type;
    const int ref_len = p.ref_len, max_iter = p.max_iter;
    const double* __restrict__ re = b.ref_re;
    const double* __restrict__ im = b.ref_im;
    const double dcy = (p.ref_py - sub_j) * p.dy_hi;
    const double dcx = (sub_i - p.ref_px) * p.dx_hi;
    double dzx = 0.0, dzy = 0.0;
    int k = 0;
    if (p.bbsa_skip > 0 && ft != 1) {
        const double ux = dcx * p.bbsa_inv_r, uy = dcy * p.bbsa_inv_r;
        if (ux * ux + uy * uy <= 1.0) {
            const cplx d = bbsa_eval(p.bbsa, ux, uy);
            dzx = d.r;
            dzy = d.i;
            k = p.bbsa_skip;
        }
    }
    const int k0 = k;
    int m = k, leaps = 0, skipped = 0;
    auto done = [&](SampleOut o, int k_end) {
        o.iters = k_end - k0 - skipped;
        o.iters2 = 0;
        o.leaps = leaps;
        return o;
    };
    const int levels = p.bla_levels;
    const bool has_bla = levels > 1 && b.bla != nullptr && (ft == 0 || ft == 4);
    const size_t L = (size_t)ref_len;
    const double inv_ln = inv_ln_for(ft, p.gen_n);
    while (k < max_iter) {
        const double rx = __ldg(re + m), ry = __ldg(im + m);
        const double zx = rx + dzx, zy = ry + dzy;
        const double mag2 = fast ? fma(zx, zx, zy * zy) : zx * zx + zy * zy;
        if (!(mag2 <= kBailout)) {
            if (isnan(mag2)) return done(glitch_sample(k), k);
            return done(escaped_sample(k, mag2, inv_ln), k);
        }
        const double dz_mag2 = fast ? fma(dzx, dzx, dzy * dzy) : dzx * dzx + dzy * dzy;
        if (mag2 < dz_mag2 || (m == ref_len && m > 0)) {
            dzx = zx;
            dzy = zy;
            m = 0;
            continue;
        }
        if (has_bla && m < ref_len - 1 && dz_mag2 < __ldg(b.bla + (size_t)m * 5 + 4)) {
            int best = 0, max_d = levels - 1;
            if (dz_mag2 == 0.0 && (dzx != 0.0 || dzy != 0.0)) max_d = min(max_d, 8);
            max_d = min(max_d, 31 - __clz(max_iter - k));
            for (int d = max_d; d > 0; --d) {
                if (m + (1 << d) < ref_len && dz_mag2 < __ldg(b.bla + ((size_t)d * L + m) * 5 + 4)) {
                    best = d;
                    break;
                }
            }
            const double* e = b.bla + ((size_t)best * L + m) * 5;
            const double ar = __ldg(e), ai = __ldg(e + 1), br = __ldg(e + 2), bi = __ldg(e + 3);
            double nx, ny;
            if (kCpu) {
                nx = (ar * dzx - ai * dzy) + (br * dcx - bi * dcy);
                ny = (ar * dzy + ai * dzx) + (br * dcy + bi * dcx);
            } else {
                nx = fma(ar, dzx, fma(-ai, dzy, fma(br, dcx, -bi * dcy)));
                ny = fma(ar, dzy, fma(ai, dzx, fma(br, dcy, bi * dcx)));
            }
            dzx = nx;
            dzy = ny;
            if (isnan(dzx) || isnan(dzy) || isinf(dzx) || isinf(dzy)) return done(glitch_sample(k), k);
            m += 1 << best;
            k += 1 << best;
            ++leaps;
            skipped += 1 << best;
            continue;
        }
        if (ft == 0) {
            double nx, ny;
            if (fast) {
                const double ax = fma(2.0, rx, dzx), ay = fma(2.0, ry, dzy);
                nx = fma(ax, dzx, fma(-ay, dzy, dcx));
                ny = fma(ax, dzy, fma(ay, dzx, dcy));
            } else if (kCpu) {
                nx = (2.0 * rx + dzx) * dzx - (2.0 * ry + dzy) * dzy + dcx;
                ny = 2.0 * ((rx + dzx) * dzy + ry * dzx) + dcy;
            } else {
                nx = fma(2.0 * rx + dzx, dzx, fma(-(2.0 * ry + dzy), dzy, dcx));
                ny = fma(2.0, fma(rx + dzx, dzy, ry * dzx), dcy);
            }
            dzx = nx;
            dzy = ny;
        } else if (ft == 1) {
            const double nx = (2.0 * rx + dzx) * dzx - (2.0 * ry + dzy) * dzy + dcx;
            const double sx = rx >= 0.0 ? 1.0 : -1.0, sy = ry >= 0.0 ? 1.0 : -1.0;
            const double ddx = (rx + dzx) * sx >= 0.0 ? sx * dzx : -sx * (2.0 * rx + dzx);
            const double ddy = (ry + dzy) * sy >= 0.0 ? sy * dzy : -sy * (2.0 * ry + dzy);
            dzy = 2.0 * (fabs(rx) * ddy + fabs(ry) * ddx + ddx * ddy) - dcy;
            dzx = nx;
        } else {
            double pr = dzx, pi = dzy, qr = rx, qi = ry;
            for (int t = 0; t < p.gen_n - 1; ++t) {
                const cplx t1 = cmul(pr, pi, rx, ry);
                const cplx t2 = cmul(pr + qr, pi + qi, dzx, dzy);
                pr = t1.r + t2.r;
                pi = t1.i + t2.i;
                const cplx q = cmul(qr, qi, rx, ry);
                qr = q.r;
                qi = q.i;
            }
            const cplx kz = cmul(p.gen_kr, p.gen_ki, dzx, dzy);
            dzx = pr + kz.r + dcx;
            dzy = pi + kz.i + dcy;
        }
        ++m;
        ++k;
    }
    return done(interior_sample(), max_iter);
}

template <int ARITH>
__device__ __forceinline__ SampleOut perturb_sample_at(const ApFrameParams& p,
                                                       const ApFrameBuffers& b, double sub_i,
                                                       double sub_j) {
    if (p.flags & AP_FLAG_REBASE) return rebase_sample_at<ARITH>(p, b, sub_i, sub_j);
    constexpr bool kCpu = (ARITH == AP_ARITH_REF_CPU);
    const int ft = p.fractal_type;
    const bool julia = (ft == 2 || ft == 3);
    const int ref_len = p.ref_len, max_iter = p.max_iter;
    const double* __restrict__ re = b.ref_re;
    const double* __restrict__ im = b.ref_im;
    const bool strict = p.strict_glitch > 0;
    const double dcy = (p.ref_py - sub_j) * p.dy_hi;
    const double dcx = (sub_i - p.ref_px) * p.dx_hi;

    double dzx, dzy;
    int k;
    bool series = false;
    if (p.bbsa_skip > 0 && (ft == 0 || ft == 2 || ft == 4)) {
        const double ux = dcx * p.bbsa_inv_r, uy = dcy * p.bbsa_inv_r;
        if (ux * ux + uy * uy <= 1.0) {
            const cplx d = bbsa_eval(p.bbsa, ux, uy);
            dzx = d.r;
            dzy = d.i;
            k = p.bbsa_skip;
            series = true;
        }
    }
    if (!series) {
        dzx = julia ? dcx : 0.0;
        dzy = julia ? dcy : 0.0;
        k = 0;
    }
    const double dcpx = julia ? 0.0 : dcx, dcpy = julia ? 0.0 : dcy;
    int glitch = 0;
    const int k0 = k;
    int leaps = 0, skipped = 0, k2 = -1;
    auto done = [&](SampleOut o, int k_end) {
        o.iters = (k2 < 0 ? k_end - k0 : k2 - k0) - skipped;
        o.iters2 = k2 < 0 ? 0 : k_end - k2;
        o.leaps = leaps;
        return o;
    };
    const int levels = p.bla_levels;
    const bool has_bla = levels > 1 && b.bla != nullptr && (ft == 0 || ft == 2 || ft == 4);
    const size_t L = (size_t)ref_len;
    const double inv_ln = inv_ln_for(ft, p.gen_n);

    while (k < ref_len) {
        const double rx = __ldg(re + k), ry = __ldg(im + k);
        const double zx = rx + dzx, zy = ry + dzy;
        const double mag2 = zx * zx + zy * zy;
        if (mag2 > kBailout) {
            if ((p.flags & AP_FLAG_ESCAPE_GLITCH) && strict && k > 15 && (rx * rx + ry * ry) < 4.0)
                glitch = 1;
            SampleOut o = escaped_sample(k, mag2, inv_ln);
            o.glitch = glitch;
            return done(o, k);
        }
        if (strict && k > 15) {
            const double r_mag2 = rx * rx + ry * ry;
            if (mag2 < 1e-6 * r_mag2 && r_mag2 > 1e-8) glitch = 1;
        }
        if (has_bla && k < ref_len - 1) {
            const double dz_mag2 = dzx * dzx + dzy * dzy;
            if (dz_mag2 < __ldg(b.bla + (size_t)k * 5 + 4)) {
                int best = 0, max_d = levels - 1;
                if (dz_mag2 == 0.0 && (dzx != 0.0 || dzy != 0.0)) max_d = min(max_d, 8);
                for (int d = max_d; d > 0; --d) {
                    if (k + (1 << d) < ref_len &&
                        dz_mag2 < __ldg(b.bla + ((size_t)d * L + k) * 5 + 4)) {
                        best = d;
                        break;
                    }
                }
                const double* e = b.bla + ((size_t)best * L + k) * 5;
                const double ar = __ldg(e), ai = __ldg(e + 1), br = __ldg(e + 2), bi = __ldg(e + 3);
                double nx, ny;
                if (kCpu) {
                    nx = (ar * dzx - ai * dzy) + (br * dcpx - bi * dcpy);
                    ny = (ar * dzy + ai * dzx) + (br * dcpy + bi * dcpx);
                } else {
                    nx = fma(ar, dzx, fma(-ai, dzy, fma(br, dcpx, -bi * dcpy)));
                    ny = fma(ar, dzy, fma(ai, dzx, fma(br, dcpy, bi * dcpx)));
                }
                dzx = nx;
                dzy = ny;
                if (isnan(dzx) || isnan(dzy) || isinf(dzx) || isinf(dzy)) return done(glitch_sample(k), k);
                k += 1 << best;
                ++leaps;
                skipped += 1 << best;
                continue;
            }
        }
        if (ft == 0 || ft == 2) {
            double nx, ny;
            if (kCpu) {
                nx = (2.0 * rx + dzx) * dzx - (2.0 * ry + dzy) * dzy + dcpx;
                ny = 2.0 * ((rx + dzx) * dzy + ry * dzx) + dcpy;
            } else {
                nx = fma(2.0 * rx + dzx, dzx, fma(-(2.0 * ry + dzy), dzy, dcpx));
                ny = fma(2.0, fma(rx + dzx, dzy, ry * dzx), dcpy);
            }
            dzx = nx;
            dzy = ny;
        } else if (ft == 1 || ft == 3) {
            const double nx = (2.0 * rx + dzx) * dzx - (2.0 * ry + dzy) * dzy + dcpx;
            const double sx = rx >= 0.0 ? 1.0 : -1.0, sy = ry >= 0.0 ? 1.0 : -1.0;
            const double ddx = (rx + dzx) * sx >= 0.0 ? sx * dzx : -sx * (2.0 * rx + dzx);
            const double ddy = (ry + dzy) * sy >= 0.0 ? sy * dzy : -sy * (2.0 * ry + dzy);
            dzy = 2.0 * (fabs(rx) * ddy + fabs(ry) * ddx + ddx * ddy) - dcpy;
            dzx = nx;
        } else {
            double pr = dzx, pi = dzy, qr = rx, qi = ry;
            for (int t = 0; t < p.gen_n - 1; ++t) {
                const cplx t1 = cmul(pr, pi, rx, ry);
                const cplx t2 = cmul(pr + qr, pi + qi, dzx, dzy);
                pr = t1.r + t2.r;
                pi = t1.i + t2.i;
                const cplx q = cmul(qr, qi, rx, ry);
                qr = q.r;
                qi = q.i;
            }
            const cplx kz = cmul(p.gen_kr, p.gen_ki, dzx, dzy);
            dzx = pr + kz.r + dcpx;
            dzy = pi + kz.i + dcpy;
        }
        ++k;
    }

    // Stage 2: past the end of the reference orbit, iterate z directly.
    double zx = __ldg(re + ref_len) + dzx, zy = __ldg(im + ref_len) + dzy;
    const double cx = julia ? p.julia_cx_hi : p.ref_cx + dcx;
    const double cy = julia ? p.julia_cy_hi : p.ref_cy + dcy;
    if (ref_len < max_iter) glitch = 1;
    k2 = k;
    const bool nan_guard = (p.flags & AP_FLAG_NAN_GUARD) != 0;
    while (k < max_iter) {
        const double zx2 = zx * zx, zy2 = zy * zy;
        const double mag2 = zx2 + zy2;
        if (nan_guard && (isnan(mag2) || isinf(mag2))) return done(glitch_sample(k), k);
        if (mag2 > kBailout) {
            SampleOut o = escaped_sample(k, mag2, inv_ln);
            o.glitch = glitch;
            return done(o, k);
        }
        if (ft == 0 || ft == 2) {
            zy = 2.0 * zx * zy + cy;
            zx = zx2 - zy2 + cx;
        } else if (ft == 1 || ft == 3) {
            zy = 2.0 * fabs(zx) * fabs(zy) - cy;
            zx = zx2 - zy2 + cx;
        } else {
            double zr = zx, zi = zy;
            for (int t = 0; t < p.gen_n - 1; ++t) {
                const double nr = zr * zx - zi * zy, ni = zr * zy + zi * zx;
                zr = nr;
                zi = ni;
            }
            const double kzr = p.gen_kr * zx - p.gen_ki * zy;
            const double kzi = p.gen_kr * zy + p.gen_ki * zx;
            zx = zr + kzr + cx;
            zy = zi + kzi + cy;
        }
        ++k;
    }
    SampleOut o = interior_sample();
    o.glitch = glitch;
    return done(o, max_iter);
}

// ---------------------------------------------------------------- FloatExp
// pow2_f64 of the reference (math_core/cuda_kernels.py:97-102): 2^e, the
// largest double at e >= 1023 and 0 at e <= -1022, built from its bits.
__device__ __forceinline__ double pow2_f64(int e) {
    if (e >= 1023) return 1.7976931348623157e+308;
    if (e <= -1022) return 0.0;
    return __longlong_as_double((long long)(e + 1023) << 52);
}

// Python's max(a, b) on floats: b when b > a, else a (NaN-order preserving).
__device__ __forceinline__ double py_max(double a, double b) { return b > a ? b : a; }

// Keep the mantissa pair within [2^-16, 2^16] by exact 2^16 rescaling
// (math_core/cuda_kernels.py:913-923).  The loops stop on non-finite values,
// where some reference variants would not.
__device__ __forceinline__ void renorm16(double& x, double& y, int& e) {
    double mag = py_max(fabs(x), fabs(y));
    while (mag > 65536.0 && isfinite(mag)) {
        x *= 1.52587890625e-05;
        y *= 1.52587890625e-05;
        e += 16;
        mag = py_max(fabs(x), fabs(y));
    }
    while (mag < 1.52587890625e-05 && mag > 0.0 && isfinite(mag)) {
        x *= 65536.0;
        y *= 65536.0;
        e -= 16;
        mag = py_max(fabs(x), fabs(y));
    }
}

// Pauldelbrot test on the scaled pair (check_glitch_cancellation_floatexp,
// math_core/cuda_kernels.py:105-135, cpu_kernels.py:171-201).
__device__ __forceinline__ bool floatexp_glitch(double rx, double ry, double dzx, double dzy,
                                                int eff_exp) {
    const double r_max = py_max(fabs(rx), fabs(ry));
    if (r_max < 1e-4) return false;
    const double dz_max = py_max(fabs(dzx), fabs(dzy));
    if (dz_max <= 0.0) return false;
    const int r_exp = (int)(log(r_max) * 1.4426950408889634);
    const int dz_exp = (int)(log(dz_max) * 1.4426950408889634);
    const int diff = r_exp - (eff_exp + dz_exp);
    if (diff > 10 || diff < -10) return false;
    const double scale_r = pow2_f64(-r_exp), scale_dz = pow2_f64(eff_exp - r_exp);
    const double rxs = rx * scale_r, rys = ry * scale_r;
    const double zx = rxs + dzx * scale_dz, zy = rys + dzy * scale_dz;
    return zx * zx + zy * zy < 1e-6 * (rxs * rxs + rys * rys);
}

// FloatExp perturbation: the true delta is (dzx, dzy) 2^(z_exp - E) with the
// mantissa pair kept in [2^-16, 2^16]; delta_c = dc_norm 2^-E (dx/dy are the
// normalised spacings).  Semantics of cpu_compute_perturbation_sample_floatexp
// (math_core/cpu_kernels.py:606-1021) and of the CUDA variants
// compute_perturbation_sample_floatexp[_bla] (math_core/cuda_kernels.py:819-1499):
// they differ in the Burning Ship delta form (ARITH), the BLA leap's fused
// multiply-adds (ARITH) and the stage-2 NaN guard (AP_FLAG_NAN_GUARD).  BBSA
// starts are never used: the reference maps orders 4/8 to chained BLA here.
template <int ARITH>
__device__ __forceinline__ SampleOut floatexp_sample_at(const ApFrameParams& p,
                                                        const ApFrameBuffers& b, double sub_i,
                                                        double sub_j) {
    constexpr bool kCpu = (ARITH == AP_ARITH_REF_CPU);
    const int ft = p.fractal_type;
    const bool julia = (ft == 2 || ft == 3);
    const int ref_len = p.ref_len, max_iter = p.max_iter, E = p.e_scale;
    const double* __restrict__ re = b.ref_re;
    const double* __restrict__ im = b.ref_im;
    const bool strict = p.strict_glitch > 0;
    const double dcy = (p.ref_py - sub_j) * p.dy_hi;
    const double dcx = (sub_i - p.ref_px) * p.dx_hi;
    double dzx = julia ? dcx : 0.0, dzy = julia ? dcy : 0.0;
    int z_exp = 0, k = 0;
    const double dcpx = julia ? 0.0 : dcx, dcpy = julia ? 0.0 : dcy;
    int glitch = 0, leaps = 0, skipped = 0, k2 = -1;
    auto done = [&](SampleOut o, int k_end) {
        o.iters = (k2 < 0 ? k_end : k2) - skipped;
        o.iters2 = k2 < 0 ? 0 : k_end - k2;
        o.leaps = leaps;
        return o;
    };
    const int levels = p.bla_levels;
    const bool has_bla = levels > 1 && b.bla != nullptr && (ft == 0 || ft == 2 || ft == 4);
    const size_t L = (size_t)ref_len;
    const double inv_ln = inv_ln_for(ft, p.gen_n);

    while (k < ref_len) {
        const double rx = __ldg(re + k), ry = __ldg(im + k);
        const int eff_exp = z_exp - E;
        if (eff_exp >= -50) {
            const double sc = pow2_f64(eff_exp);
            const double zx = rx + dzx * sc, zy = ry + dzy * sc;
            const double mag2 = zx * zx + zy * zy;
            if (mag2 > kBailout) {
                SampleOut o = escaped_sample(k, mag2, inv_ln);
                o.glitch = glitch;
                return done(o, k);
            }
        }
        if (strict && k > 15 && floatexp_glitch(rx, ry, dzx, dzy, eff_exp)) glitch = 1;

        if (has_bla && k < ref_len - 1) {
            // |delta|^2 against r^2 in scaled form, or via square roots far below 2^-510
            const int shift_r = eff_exp;
            const bool scaled = shift_r >= -510;
            double dz_mag2 = 0.0, dz_lin = 0.0;
            if (scaled) {
                const double sr = pow2_f64(shift_r);
                dz_mag2 = (dzx * dzx + dzy * dzy) * (sr * sr);
            } else {
                dz_lin = sqrt(dzx * dzx + dzy * dzy) * pow2_f64(max(-1020, shift_r));
            }
            auto fits = [&](double r_sq) {
                return scaled ? (dz_mag2 < r_sq) : (r_sq > 0.0 && dz_lin < sqrt(r_sq));
            };
            if (fits(__ldg(b.bla + (size_t)k * 5 + 4))) {
                int best = 0;
                for (int d = levels - 1; d > 0; --d) {
                    if (k + (1 << d) < ref_len && fits(__ldg(b.bla + ((size_t)d * L + k) * 5 + 4))) {
                        best = d;
                        break;
                    }
                }
                const double* e = b.bla + ((size_t)best * L + k) * 5;
                const double ar = __ldg(e), ai = __ldg(e + 1), br = __ldg(e + 2), bi = __ldg(e + 3);
                const double scale_c = (z_exp >= -1020 && z_exp <= 1020) ? pow2_f64(-z_exp) : 0.0;
                const double cxs = dcpx * scale_c, cys = dcpy * scale_c;
                double nx, ny;
                if (kCpu) {
                    nx = (ar * dzx - ai * dzy) + (br * cxs - bi * cys);
                    ny = (ar * dzy + ai * dzx) + (br * cys + bi * cxs);
                } else {
                    nx = fma(ar, dzx, fma(-ai, dzy, fma(br, cxs, -bi * cys)));
                    ny = fma(ar, dzy, fma(ai, dzx, fma(br, cys, bi * cxs)));
                }
                dzx = nx;
                dzy = ny;
                if (isnan(dzx) || isnan(dzy) || isinf(dzx) || isinf(dzy)) return done(glitch_sample(k), k);
                renorm16(dzx, dzy, z_exp);
                k += 1 << best;
                ++leaps;
                skipped += 1 << best;
                continue;
            }
        }

        const int shift_nl = z_exp - E;
        const double scale_c = (z_exp >= -1020 && z_exp <= 1020) ? pow2_f64(-z_exp) : 0.0;
        if (ft == 0 || ft == 2) {
            double lx = 2.0 * (rx * dzx - ry * dzy);
            double ly = 2.0 * (rx * dzy + ry * dzx);
            if (shift_nl >= -1020) {
                const double sn = pow2_f64(shift_nl);
                lx += (dzx * dzx - dzy * dzy) * sn;
                ly += (2.0 * dzx * dzy) * sn;
            }
            dzx = lx + dcpx * scale_c;
            dzy = ly + dcpy * scale_c;
        } else if (ft == 1 || ft == 3) {
            const double sn = shift_nl >= -1020 ? pow2_f64(shift_nl) : 0.0;
            const double sx = rx >= 0.0 ? 1.0 : -1.0, sy = ry >= 0.0 ? 1.0 : -1.0;
            if (kCpu) {  // math_core/cpu_kernels.py:795-829
                const double se = eff_exp >= -1020 ? pow2_f64(eff_exp) : 0.0;
                const double inv = eff_exp <= 1020 ? pow2_f64(-eff_exp) : 0.0;
                double fx, ex, fy, ey;
                if ((rx + dzx * se) * sx >= 0.0) { fx = sx; ex = 0.0; }
                else { fx = -sx; ex = eff_exp <= 1020 ? ((-sx * 2.0) * rx) * inv : 0.0; }
                if ((ry + dzy * se) * sy >= 0.0) { fy = sy; ey = 0.0; }
                else { fy = -sy; ey = eff_exp <= 1020 ? ((-sy * 2.0) * ry) * inv : 0.0; }
                const double lx = (2.0 * rx + dzx * sn) * dzx - (2.0 * ry + dzy * sn) * dzy + dcpx * scale_c;
                const double dxn = fx * dzx + ex, dyn = fy * dzy + ey;
                const double ly = 2.0 * (fabs(rx) * dyn + fabs(ry) * dxn + dxn * dyn * sn) - dcpy * scale_c;
                dzx = lx;
                dzy = ly;
            } else {  // math_core/cuda_kernels.py:964-985
                const double sd = eff_exp >= -60 ? pow2_f64(eff_exp) : 0.0;
                const double inv = pow2_f64(-eff_exp);
                const double ddx = (rx + dzx * sd) * sx >= 0.0 ? sx * dzx : -sx * (2.0 * rx * inv + dzx);
                const double ddy = (ry + dzy * sd) * sy >= 0.0 ? sy * dzy : -sy * (2.0 * ry * inv + dzy);
                double lx = 2.0 * (rx * dzx - ry * dzy);
                double ly = 2.0 * (fabs(rx) * ddy + fabs(ry) * ddx);
                if (shift_nl >= -1020) {
                    lx += (dzx * dzx - dzy * dzy) * sn;
                    ly += (2.0 * ddx * ddy) * sn;
                }
                dzx = lx + dcpx * scale_c;
                dzy = ly - dcpy * scale_c;
            }
        } else {
            const double sn = shift_nl >= -1020 ? pow2_f64(shift_nl) : 0.0;
            double pr = dzx, pi = dzy, qr = rx, qi = ry;
            for (int t = 0; t < p.gen_n - 1; ++t) {
                const cplx t1 = cmul(pr, pi, rx, ry);
                const cplx t2 = cmul(qr, qi, dzx, dzy);
                const cplx t3 = cmul(pr, pi, dzx, dzy);
                pr = t1.r + t2.r + t3.r * sn;
                pi = t1.i + t2.i + t3.i * sn;
                const cplx q = cmul(qr, qi, rx, ry);
                qr = q.r;
                qi = q.i;
            }
            const cplx kz = cmul(p.gen_kr, p.gen_ki, dzx, dzy);
            dzx = pr + kz.r + dcpx * scale_c;
            dzy = pi + kz.i + dcpy * scale_c;
        }
        renorm16(dzx, dzy, z_exp);
        ++k;
    }

    // Stage 2: z = Z_ref_len + delta, then direct FP64 iteration with c = ref_c + dc.
    const int eff_exp = z_exp - E;
    const double sfb = eff_exp >= -60 ? pow2_f64(eff_exp) : 0.0;
    double zx = __ldg(re + ref_len) + dzx * sfb, zy = __ldg(im + ref_len) + dzy * sfb;
    const double scf = E <= 1020 ? pow2_f64(-E) : 0.0;
    const double cx = julia ? p.julia_cx_hi : p.ref_cx + dcpx * scf;
    const double cy = julia ? p.julia_cy_hi : p.ref_cy + dcpy * scf;
    k2 = k;
    {
        const double mag2 = zx * zx + zy * zy;
        if (mag2 > kBailout) {  // escaped together with the reference at k = ref_len
            SampleOut o = escaped_sample(ref_len, mag2, inv_ln);
            o.glitch = glitch;
            return done(o, k);
        }
    }
    if (ref_len < max_iter) glitch = 1;
    const bool nan_guard = (p.flags & AP_FLAG_NAN_GUARD) != 0;
    while (k < max_iter) {
        const double zx2 = zx * zx, zy2 = zy * zy;
        const double mag2 = zx2 + zy2;
        if (nan_guard && (isnan(mag2) || isinf(mag2))) return done(glitch_sample(k), k);
        if (mag2 > kBailout) {
            SampleOut o = escaped_sample(k, mag2, inv_ln);
            o.glitch = glitch;
            return done(o, k);
        }
        if (ft == 0 || ft == 2) {
            zy = 2.0 * zx * zy + cy;
            zx = zx2 - zy2 + cx;
        } else if (ft == 1 || ft == 3) {
            zy = 2.0 * fabs(zx) * fabs(zy) - cy;
            zx = zx2 - zy2 + cx;
        } else {
            double zr = zx, zi = zy;
            for (int t = 0; t < p.gen_n - 1; ++t) {
                const double nr = zr * zx - zi * zy, ni = zr * zy + zi * zx;
                zr = nr;
                zi = ni;
            }
            const double kzr = p.gen_kr * zx - p.gen_ki * zy;
            const double kzi = p.gen_kr * zy + p.gen_ki * zx;
            zx = zr + kzr + cx;
            zy = zi + kzi + cy;
        }
        ++k;
    }
    SampleOut o = interior_sample();
    o.glitch = glitch;
    return done(o, max_iter);
}

}  // namespace ap
