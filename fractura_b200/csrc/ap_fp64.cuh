// ap_fp64.cuh -- direct FP64 escape-time iteration for the five formulas.
//
// Semantics of compute_fp64_sample (math_core/cuda_kernels.py:264-317) and
// cpu_compute_fp64_sample (math_core/cpu_kernels.py:228-266).  ARITH picks
// which multiply-adds are fused:
//   AP_ARITH_REF_CPU  the fused/reassociated forms the reference's Numba CPU
//                     build executes (bit-identical to its output);
//   AP_ARITH_REF_CUDA the reference's CUDA source expressions, unfused.
#pragma once

#include "ap_common.cuh"

namespace ap {

template <int ARITH>
__device__ __forceinline__ SampleOut fp64_sample(double x, double y, const ApFrameParams& p) {
    constexpr bool kCpu = (ARITH == AP_ARITH_REF_CPU);
    const int ft = p.fractal_type;
    const int max_iter = p.max_iter;

    if (ft == 0) {
        // Main cardioid and period-2 bulb early-out.
        const double xm = x - 0.25;
        const double y2 = y * y;
        const double q = kCpu ? fma(xm, xm, y2) : xm * xm + y2;
        const double xp = x + 1.0;
        const double b = kCpu ? fma(xp, xp, y2) : xp * xp + y2;
        if ((q * (q + xm) <= 0.25 * y2) || (b <= 0.0625)) return skipped_sample();
    }
    double zx, zy, cx, cy;
    if (ft == 2 || ft == 3) {
        zx = x; zy = y; cx = p.julia_cx_hi; cy = p.julia_cy_hi;
    } else {
        zx = 0.0; zy = 0.0; cx = x; cy = y;
    }

    if (ft == 0 || ft == 2) {
        for (int k = 0; k < max_iter; ++k) {
            const double zx2 = zx * zx, zy2 = zy * zy;
            const double mag2 = zx2 + zy2;
            if (mag2 > kBailout) return escaped_sample(k, mag2, kInvLn2);
            if (kCpu) {
                const double nzy = fma(zy + zy, zx, cy);
                zx = (cx - zy2) + zx2;
                zy = nzy;
            } else {
                zy = 2.0 * zx * zy + cy;
                zx = zx2 - zy2 + cx;
            }
        }
        return interior_after(max_iter);
    }
    if (ft == 1 || ft == 3) {
        for (int k = 0; k < max_iter; ++k) {
            const double zx2 = zx * zx, zy2 = zy * zy;
            const double mag2 = zx2 + zy2;
            if (mag2 > kBailout) return escaped_sample(k, mag2, kInvLn2);
            const double ax = fabs(zx), ay = fabs(zy);
            if (kCpu) {
                const double nzy = fma(ax, ay + ay, -cy);
                zx = (cx + zx2) - zy2;
                zy = nzy;
            } else {
                zy = 2.0 * ax * ay - cy;
                zx = zx2 - zy2 + cx;
            }
        }
        return interior_after(max_iter);
    }
    if (ft == 4) {
        const int n = p.gen_n;
        const double kr = p.gen_kr, ki = p.gen_ki;
        const double inv_ln = inv_ln_for(4, n);
        for (int k = 0; k < max_iter; ++k) {
            double mag2;
            if (kCpu) {
                mag2 = fma(zx, zx, zy * zy);
            } else {
                mag2 = zx * zx + zy * zy;
            }
            if (mag2 > kBailout) return escaped_sample(k, mag2, inv_ln);
            double zr = zx, zi = zy;
            for (int t = 0; t < n - 1; ++t) {
                double nr, ni;
                if (kCpu) {
                    nr = fma(zr, zx, -(zi * zy));
                    ni = fma(zi, zx, zr * zy);
                } else {
                    nr = zr * zx - zi * zy;
                    ni = zr * zy + zi * zx;
                }
                zr = nr;
                zi = ni;
            }
            if (kCpu) {
                const double a = fma(zx, kr, -fma(ki, zy, -cx));
                const double b = fma(ki, zx, fma(zy, kr, cy));
                zx = a + zr;
                zy = b + zi;
            } else {
                const double kz_r = kr * zx - ki * zy;
                const double kz_i = kr * zy + ki * zx;
                zx = zr + kz_r + cx;
                zy = zi + kz_i + cy;
            }
        }
        return interior_after(max_iter);
    }
    return interior_sample();
}

}  // namespace ap
