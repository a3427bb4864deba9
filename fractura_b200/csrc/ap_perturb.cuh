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

template <int ARITH>
__device__ __forceinline__ SampleOut perturb_sample_at(const ApFrameParams& p,
                                                       const ApFrameBuffers& b, double sub_i,
                                                       double sub_j) {
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

template <int ARITH>
__device__ __forceinline__ SampleOut floatexp_sample_at(const ApFrameParams& p,
                                                        const ApFrameBuffers& b, double sub_i,
                                                        double sub_j) {
    (void)p; (void)b; (void)sub_i; (void)sub_j;
    return interior_sample();
}

}  // namespace ap
