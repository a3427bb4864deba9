// ap_dd.cuh -- double-double direct iteration.
//
// Semantics of compute_dd_sample (math_core/cuda_kernels.py:321-418) and
// cpu_compute_dd_sample (math_core/cpu_kernels.py:271-369).  The two
// references differ only in the error-free product: the CUDA build uses
// fma(a, b, -a*b), the CPU build a Dekker split; ARITH selects which.
#pragma once

#include "ap_common.cuh"

namespace ap {

struct dd {
    double hi, lo;
};

__device__ __forceinline__ dd two_sum(double a, double b) {
    const double s = a + b;
    const double v = s - a;
    const double e = (a - (s - v)) + (b - v);
    return {s, e};
}

template <int ARITH>
__device__ __forceinline__ dd two_prod(double a, double b) {
    if constexpr (ARITH == AP_ARITH_REF_CPU) {
        // Dekker split with 2^27 + 1 (math_core/cpu_kernels.py:104-113).
        double c = 134217729.0 * a;
        const double a_hi = c - (c - a);
        const double a_lo = a - a_hi;
        c = 134217729.0 * b;
        const double b_hi = c - (c - b);
        const double b_lo = b - b_hi;
        const double p = a * b;
        const double e = ((a_hi * b_hi - p) + a_hi * b_lo + a_lo * b_hi) + a_lo * b_lo;
        return {p, e};
    } else {
        const double p = a * b;
        return {p, fma(a, b, -p)};
    }
}

__device__ __forceinline__ dd dd_abs(dd a) {
    return (a.hi < 0.0 || (a.hi == 0.0 && a.lo < 0.0)) ? dd{-a.hi, -a.lo} : a;
}

__device__ __forceinline__ dd dd_add(dd a, dd b) {
    const dd s = two_sum(a.hi, b.hi);
    return two_sum(s.hi, s.lo + a.lo + b.lo);
}

__device__ __forceinline__ dd dd_sub(dd a, dd b) {
    const dd s = two_sum(a.hi, -b.hi);
    return two_sum(s.hi, s.lo + a.lo - b.lo);
}

template <int ARITH>
__device__ __forceinline__ dd dd_mul(dd a, dd b) {
    const dd p = two_prod<ARITH>(a.hi, b.hi);
    return two_sum(p.hi, p.lo + a.hi * b.lo + a.lo * b.hi);
}

template <int ARITH>
__device__ __forceinline__ dd dd_mul_f64(dd a, double b) {
    const dd p = two_prod<ARITH>(a.hi, b);
    return two_sum(p.hi, p.lo + a.lo * b);
}

template <int ARITH>
__device__ __forceinline__ dd dd_sqr(dd a) {
    const dd p = two_prod<ARITH>(a.hi, a.hi);
    return two_sum(p.hi, p.lo + 2.0 * a.hi * a.lo);
}

template <int ARITH>
__device__ __forceinline__ SampleOut dd_sample(dd cxv, dd cyv, const ApFrameParams& p) {
    const int ft = p.fractal_type;
    const int max_iter = p.max_iter;
    if (ft == 0) {
        const double xm = cxv.hi - 0.25;
        const double y2 = cyv.hi * cyv.hi;
        const double q = xm * xm + y2;
        if ((q * (q + xm) <= 0.25 * y2) || ((cxv.hi + 1.0) * (cxv.hi + 1.0) + y2 <= 0.0625))
            return skipped_sample();
    }
    const dd jx{p.julia_cx_hi, p.julia_cx_lo}, jy{p.julia_cy_hi, p.julia_cy_lo};
    dd zx, zy, cx, cy;
    if (ft == 2 || ft == 3) {
        zx = cxv; zy = cyv; cx = jx; cy = jy;
    } else {
        zx = {0.0, 0.0}; zy = {0.0, 0.0}; cx = cxv; cy = cyv;
    }
    if (ft == 0 || ft == 2) {
        for (int k = 0; k < max_iter; ++k) {
            const dd zx2 = dd_sqr<ARITH>(zx), zy2 = dd_sqr<ARITH>(zy);
            const double mag2 = zx2.hi + zy2.hi;
            if (mag2 > kBailout) return escaped_sample(k, mag2, kInvLn2);
            const dd sub = dd_sub(zx2, zy2);
            const dd zxy = dd_mul<ARITH>(zx, zy);
            zx = dd_add(sub, cx);
            zy = dd_add(dd{zxy.hi * 2.0, zxy.lo * 2.0}, cy);
        }
        return interior_after(max_iter);
    }
    if (ft == 1 || ft == 3) {
        for (int k = 0; k < max_iter; ++k) {
            const dd zx2 = dd_sqr<ARITH>(zx), zy2 = dd_sqr<ARITH>(zy);
            const double mag2 = zx2.hi + zy2.hi;
            if (mag2 > kBailout) return escaped_sample(k, mag2, kInvLn2);
            const dd sub = dd_sub(zx2, zy2);
            const dd zxy = dd_mul<ARITH>(dd_abs(zx), dd_abs(zy));
            zx = dd_add(sub, cx);
            zy = dd_sub(dd{zxy.hi * 2.0, zxy.lo * 2.0}, cy);
        }
        return interior_after(max_iter);
    }
    if (ft == 4) {
        const int n = p.gen_n;
        const double kr = p.gen_kr, ki = p.gen_ki;
        const double inv_ln = inv_ln_for(4, n);
        for (int k = 0; k < max_iter; ++k) {
            const dd zx2 = dd_sqr<ARITH>(zx), zy2 = dd_sqr<ARITH>(zy);
            const double mag2 = zx2.hi + zy2.hi;
            if (mag2 > kBailout) return escaped_sample(k, mag2, inv_ln);
            dd cr = zx, ci = zy;
            for (int t = 0; t < n - 1; ++t) {
                const dd re = dd_sub(dd_mul<ARITH>(cr, zx), dd_mul<ARITH>(ci, zy));
                const dd im = dd_add(dd_mul<ARITH>(cr, zy), dd_mul<ARITH>(ci, zx));
                cr = re;
                ci = im;
            }
            const dd kz_r = dd_sub(dd_mul_f64<ARITH>(zx, kr), dd_mul_f64<ARITH>(zy, ki));
            const dd kz_i = dd_add(dd_mul_f64<ARITH>(zy, kr), dd_mul_f64<ARITH>(zx, ki));
            zx = dd_add(dd_add(cr, kz_r), cx);
            zy = dd_add(dd_add(ci, kz_i), cy);
        }
        return interior_after(max_iter);
    }
    return interior_sample();
}

// Sub-sample -> DD coordinate (math_core/cuda_kernels.py:1685-1691, :1712-1719).
template <int ARITH>
__device__ __forceinline__ SampleOut dd_sample_at(const ApFrameParams& p, double sub_i,
                                                  double sub_j) {
    const dd jdy = dd_mul_f64<ARITH>(dd{p.dy_hi, p.dy_lo}, sub_j);
    const dd cy = dd_sub(dd{p.y_max_hi, p.y_max_lo}, jdy);
    const dd idx = dd_mul_f64<ARITH>(dd{p.dx_hi, p.dx_lo}, sub_i);
    const dd cx = dd_add(dd{p.x_min_hi, p.x_min_lo}, idx);
    return dd_sample<ARITH>(cx, cy, p);
}

}  // namespace ap
