// ap_bbsa.cu -- series-approximation start ("BBSA") coefficients, on the host.
//
// The per-pixel start of the perturbation tier (bbsa_skip, bbsa_inv_r and
// 16 coefficients in ApFrameParams) comes from a serial recurrence over the
// reference orbit: with u = dc / r, the delta after k steps is modelled as
// sum_j a_j u^j (j = 1..4 or 1..8) and the coefficients are advanced one orbit
// step at a time until the truncation estimate exceeds the tolerance or the
// linear term exceeds 1/2.  This is _jit_compute_bbsa_coeffs
// (math_core/high_precision.py:50-530) for Mandelbrot, Julia and Multibrot
// n = 3 at orders 4 and 8 (any order other than 4 selects 8); every other case
// returns skip 0.  One dependent chain of complex
// products per orbit step, computed once per reference orbit: it runs on the
// host, beside the orbit it reads, and takes microseconds per thousand steps.
#include <cmath>
#include <cstring>

#include "ap_common.cuh"

namespace {

// The reference advances the coefficients in a fast-math kernel.  Its compiled form
// reassociates the sums, fuses products into multiply-adds, doubles by x + x and
// drops the NaN/Inf breaks: a NaN |a_1|^2 skips the tolerance test and the step is
// kept.  Each loop below performs exactly those roundings in that order (one const
// per rounded value, std::fma where the kernel fuses; the library is compiled with
// contraction off), so the skip and all coefficients equal the reference's bit for
// bit.  With u = dc / r the delta after k steps is sum_j a_j u^j; a step is taken
// while |truncation estimate| / |a_1| <= tol and |a_1| <= 1/2.
inline void finish(int skip, int ref_len, const double* a, int n, double* out) {
    const int cap = ref_len - 2;
    out[0] = (double)(skip < cap ? skip : cap);
    for (int j = 0; j < n; ++j) out[1 + j] = a[j];
}

// Mandelbrot / Julia, order 8 (math_core/high_precision.py:82-210).
int series_quadratic8(const double* re, const double* im, int ref_len, double r, int ft, double kr, double ki,
           double tol, double* out) {
    double a1r = ft == 0 ? 0.0 : r, a1i = 0.0, a2r = 0.0, a2i = 0.0;
    double a3r = 0.0, a3i = 0.0, a4r = 0.0, a4i = 0.0;
    double a5r = 0.0, a5i = 0.0, a6r = 0.0, a6i = 0.0;
    double a7r = 0.0, a7i = 0.0, a8r = 0.0, a8i = 0.0;
    const double cc = ft == 0 ? r : 0.0;
    (void)kr;
    (void)ki;
    int k = 0;
    for (; k < ref_len; ++k) {
        const double x = re[k], y = im[k];
        const double c1r = x + x;
        const double c1i = y + y;
        const double n1r = std::fma(c1r, a1r, -(c1i * a1i)) + cc;
        const double n1i = std::fma(c1i, a1r, c1r * a1i);
        const double mc1i = -c1i;
        const double n2r = std::fma(c1r, a2r, std::fma(a1r, a1r, std::fma(mc1i, a2i, -(a1i * a1i))));
        const double n2i = std::fma(c1i, a2r, std::fma(c1r, a2i, a1i * (a1r + a1r)));
        const double t0 = std::fma(a1r, a2r, -(a1i * a2i));
        const double n3r = std::fma(-a3i, c1i, std::fma(c1r, a3r, t0 + t0));
        const double t1 = std::fma(a1r, a2i, a1i * a2r);
        const double n3i = std::fma(c1i, a3r, std::fma(c1r, a3i, t1 + t1));
        const double n4r = std::fma(c1r, a4r, std::fma(-2.0, std::fma(-a1r, a3r, a1i * a3i), std::fma(a2r, a2r, std::fma(mc1i, a4i, -(a2i * a2i)))));
        const double t2 = std::fma(a1r, a3i, std::fma(a1i, a3r, a2r * a2i));
        const double n4i = std::fma(c1i, a4r, std::fma(c1r, a4i, t2 + t2));
        const double t3 = -a1i;
        const double t4 = std::fma(a1r, a4r, std::fma(a2r, a3r, std::fma(t3, a4i, -(a2i * a3i))));
        const double n5r = std::fma(-a5i, c1i, std::fma(c1r, a5r, t4 + t4));
        const double t5 = std::fma(a1r, a4i, std::fma(a1i, a4r, std::fma(a2r, a3i, a2i * a3r)));
        const double n5i = std::fma(c1i, a5r, std::fma(c1r, a5i, t5 + t5));
        const double n6r = std::fma(c1r, a6r, std::fma(2.0, std::fma(a1r, a5r, std::fma(a2r, a4r, std::fma(t3, a5i, -(a2i * a4i)))), std::fma(a3r, a3r, std::fma(mc1i, a6i, -(a3i * a3i)))));
        const double t6 = std::fma(a1r, a5i, std::fma(a1i, a5r, std::fma(a2r, a4i, std::fma(a2i, a4r, a3r * a3i))));
        const double n6i = std::fma(c1i, a6r, std::fma(c1r, a6i, t6 + t6));
        const double t7 = std::fma(a1r, a6r, std::fma(a2r, a5r, std::fma(a3r, a4r, std::fma(t3, a6i, -std::fma(a2i, a5i, a3i * a4i)))));
        const double n7r = std::fma(-a7i, c1i, std::fma(c1r, a7r, t7 + t7));
        const double t8 = std::fma(a1r, a6i, std::fma(a1i, a6r, std::fma(a2r, a5i, std::fma(a2i, a5r, std::fma(a3r, a4i, a3i * a4r)))));
        const double n7i = std::fma(c1i, a7r, std::fma(c1r, a7i, t8 + t8));
        const double n8r = std::fma(2.0, std::fma(a1r, a7r, std::fma(a2r, a6r, std::fma(a3r, a5r, std::fma(t3, a7i, -std::fma(a2i, a6i, a3i * a5i))))), -std::fma(-a4r, a4r, a4i * a4i)) + std::fma(c1r, a8r, -(c1i * a8i));
        const double t9 = std::fma(a1r, a7i, std::fma(a1i, a7r, std::fma(a2r, a6i, std::fma(a2i, a6r, std::fma(a3r, a5i, std::fma(a3i, a5r, a4i * a4r))))));
        const double n8i = std::fma(c1i, a8r, std::fma(c1r, a8i, t9 + t9));
        const double mag_a2 = std::fma(n1r, n1r, n1i * n1i);
        if (mag_a2 > 0.0) {
            const double mag_a = std::sqrt(mag_a2);
            const double t10 = std::fma(a1r, a8r, std::fma(a2r, a7r, std::fma(a3r, a6r, std::fma(a4r, a5r, std::fma(t3, a8i, -std::fma(a2i, a7i, std::fma(a3i, a6i, a4i * a5i)))))));
            const double t11 = t10 + t10;
            const double t12 = std::fma(a1r, a8i, std::fma(a1i, a8r, std::fma(a2r, a7i, std::fma(a2i, a7r, std::fma(a3r, a6i, std::fma(a3i, a6r, std::fma(a4r, a5i, a4i * a5r)))))));
            const double t13 = t12 + t12;
            const double err = std::fma(std::sqrt(std::fma(n8r, n8r, n8i * n8i)), 0.1, std::sqrt(std::fma(t11, t11, t13 * t13)));
            if (err / mag_a > tol || mag_a > 0.5) break;
        }
        a1r = n1r; a1i = n1i; a2r = n2r; a2i = n2i;
        a3r = n3r; a3i = n3i; a4r = n4r; a4i = n4i;
        a5r = n5r; a5i = n5i; a6r = n6r; a6i = n6i;
        a7r = n7r; a7i = n7i; a8r = n8r; a8i = n8i;
    }
    const double a[16] = {a1r, a1i, a2r, a2i, a3r, a3i, a4r, a4i, a5r, a5i, a6r, a6i, a7r, a7i, a8r, a8i};
    finish(k, ref_len, a, 16, out);
    return AP_OK;
}

// Mandelbrot / Julia, order 4 (math_core/high_precision.py:211-284).
int series_quadratic4(const double* re, const double* im, int ref_len, double r, int ft, double kr, double ki,
           double tol, double* out) {
    double a1r = ft == 0 ? 0.0 : r, a1i = 0.0, a2r = 0.0, a2i = 0.0;
    double a3r = 0.0, a3i = 0.0, a4r = 0.0, a4i = 0.0;
    const double cc = ft == 0 ? r : 0.0;
    (void)kr;
    (void)ki;
    int k = 0;
    for (; k < ref_len; ++k) {
        const double x = re[k], y = im[k];
        const double c1r = x + x;
        const double c1i = y + y;
        const double n1r = cc + std::fma(c1r, a1r, -(c1i * a1i));
        const double n1i = std::fma(c1i, a1r, c1r * a1i);
        const double n2r = std::fma(c1r, a2r, std::fma(a1r, a1r, std::fma(-c1i, a2i, -(a1i * a1i))));
        const double n2i = std::fma(c1i, a2r, std::fma(c1r, a2i, a1i * (a1r + a1r)));
        const double t0 = std::fma(a1r, a2r, -(a1i * a2i));
        const double n3r = std::fma(-a3i, c1i, std::fma(c1r, a3r, t0 + t0));
        const double t1 = std::fma(a1r, a2i, a1i * a2r);
        const double n3i = std::fma(c1i, a3r, std::fma(c1r, a3i, t1 + t1));
        const double n4r = std::fma(-std::fma(-a1r, a3r, a1i * a3i), 2.0, -std::fma(-a2r, a2r, a2i * a2i)) + std::fma(c1r, a4r, -(c1i * a4i));
        const double t2 = std::fma(a1r, a3i, std::fma(a1i, a3r, a2r * a2i));
        const double n4i = std::fma(c1i, a4r, std::fma(c1r, a4i, t2 + t2));
        const double mag_a2 = std::fma(n1r, n1r, n1i * n1i);
        if (mag_a2 > 0.0) {
            const double mag_a = std::sqrt(mag_a2);
            const double t3 = std::fma(a1r, a4r, std::fma(a2r, a3r, std::fma(-a1i, a4i, -(a2i * a3i))));
            const double t4 = t3 + t3;
            const double t5 = std::fma(a1r, a4i, std::fma(a1i, a4r, std::fma(a2r, a3i, a2i * a3r)));
            const double t6 = t5 + t5;
            const double err = std::fma(std::sqrt(std::fma(n4r, n4r, n4i * n4i)), 0.1, std::sqrt(std::fma(t4, t4, t6 * t6)));
            if (err / mag_a > tol || mag_a > 0.5) break;
        }
        a1r = n1r; a1i = n1i; a2r = n2r; a2i = n2i;
        a3r = n3r; a3i = n3i; a4r = n4r; a4i = n4i;
    }
    const double a[8] = {a1r, a1i, a2r, a2i, a3r, a3i, a4r, a4i};
    finish(k, ref_len, a, 8, out);
    return AP_OK;
}

// Multibrot n = 3, order 8 (math_core/high_precision.py:286-448).
int series_cubic8(const double* re, const double* im, int ref_len, double r, int ft, double kr, double ki,
           double tol, double* out) {
    double a1r = 0.0, a1i = 0.0, a2r = 0.0, a2i = 0.0;
    double a3r = 0.0, a3i = 0.0, a4r = 0.0, a4i = 0.0;
    double a5r = 0.0, a5i = 0.0, a6r = 0.0, a6i = 0.0;
    double a7r = 0.0, a7i = 0.0, a8r = 0.0, a8i = 0.0;
    const double cc = r;
    int k = 0;
    for (; k < ref_len; ++k) {
        const double x = re[k], y = im[k];
        const double c1r = std::fma(-3.0, std::fma(-x, x, y * y), kr);
        const double c1i = std::fma(y, x * 6.0, ki);
        const double n1r = std::fma(c1r, a1r, -(c1i * a1i)) + cc;
        const double n1i = std::fma(c1r, a1i, c1i * a1r);
        const double c2r = x * 3.0;
        const double q2r = std::fma(a1r, a1r, -(a1i * a1i));
        const double mc1i = -c1i;
        const double c2i = y * 3.0;
        const double q2i = a1i * (a1r + a1r);
        const double n2r = std::fma(c1r, a2r, std::fma(c2r, q2r, std::fma(mc1i, a2i, -(c2i * q2i))));
        const double n2i = std::fma(c1r, a2i, std::fma(c1i, a2r, std::fma(c2i, q2r, c2r * q2i)));
        const double t0 = std::fma(a1r, a2r, -(a1i * a2i));
        const double t1 = t0 + t0;
        const double t2 = std::fma(a1r, a2i, a1i * a2r);
        const double t3 = t2 + t2;
        const double n3r = std::fma(c1r, a3r, std::fma(c2r, t1, std::fma(q2r, a1r, std::fma(mc1i, a3i, -std::fma(c2i, t3, q2i * a1i)))));
        const double n3i = std::fma(c1r, a3i, std::fma(c1i, a3r, std::fma(c2i, t1, std::fma(c2r, t3, std::fma(q2r, a1i, q2i * a1r)))));
        const double t4 = std::fma(-2.0, std::fma(-a1r, a3r, a1i * a3i), -std::fma(-a2r, a2r, a2i * a2i));
        const double t5 = std::fma(a1r, a3i, std::fma(a1i, a3r, a2r * a2i));
        const double t6 = t5 + t5;
        const double n4r = std::fma(c1r, a4r, std::fma(t4, c2r, std::fma(t1, a1r, std::fma(q2r, a2r, std::fma(mc1i, a4i, -std::fma(c2i, t6, std::fma(t3, a1i, q2i * a2i)))))));
        const double n4i = std::fma(c1r, a4i, std::fma(c1i, a4r, std::fma(c2i, t4, std::fma(c2r, t6, std::fma(t1, a1i, std::fma(t3, a1r, std::fma(q2r, a2i, q2i * a2r)))))));
        const double t7 = -a1i;
        const double t8 = std::fma(a1r, a4r, std::fma(a2r, a3r, std::fma(t7, a4i, -(a2i * a3i))));
        const double t9 = t8 + t8;
        const double t10 = std::fma(a1r, a4i, std::fma(a1i, a4r, std::fma(a2r, a3i, a2i * a3r)));
        const double t11 = t10 + t10;
        const double n5r = std::fma(c1r, a5r, std::fma(t4, a1r, std::fma(c2r, t9, std::fma(t1, a2r, std::fma(q2r, a3r, std::fma(mc1i, a5i, -std::fma(c2i, t11, std::fma(t3, a2i, std::fma(t6, a1i, q2i * a3i)))))))));
        const double n5i = std::fma(c1r, a5i, std::fma(c1i, a5r, std::fma(c2i, t9, std::fma(t4, a1i, std::fma(c2r, t11, std::fma(t6, a1r, std::fma(t1, a2i, std::fma(t3, a2r, std::fma(q2r, a3i, q2i * a3r)))))))));
        const double t12 = std::fma(2.0, std::fma(a1r, a5r, std::fma(a2r, a4r, std::fma(t7, a5i, -(a2i * a4i)))), -std::fma(-a3r, a3r, a3i * a3i));
        const double t13 = std::fma(a1r, a5i, std::fma(a1i, a5r, std::fma(a2r, a4i, std::fma(a2i, a4r, a3r * a3i))));
        const double t14 = t13 + t13;
        const double n6r = std::fma(c1r, a6r, std::fma(t12, c2r, std::fma(t4, a2r, std::fma(t9, a1r, std::fma(t1, a3r, std::fma(q2r, a4r, std::fma(mc1i, a6i, -std::fma(c2i, t14, std::fma(t3, a3i, std::fma(t6, a2i, std::fma(a1i, t11, q2i * a4i)))))))))));
        const double n6i = std::fma(c1r, a6i, std::fma(c1i, a6r, std::fma(c2i, t12, std::fma(t4, a2i, std::fma(c2r, t14, std::fma(t9, a1i, std::fma(t11, a1r, std::fma(t6, a2r, std::fma(t1, a3i, std::fma(t3, a3r, std::fma(q2r, a4i, q2i * a4r)))))))))));
        const double t15 = std::fma(a1r, a6r, std::fma(a2r, a5r, std::fma(a3r, a4r, std::fma(t7, a6i, -std::fma(a2i, a5i, a3i * a4i)))));
        const double t16 = t15 + t15;
        const double t17 = std::fma(a1r, a6i, std::fma(a1i, a6r, std::fma(a2r, a5i, std::fma(a2i, a5r, std::fma(a3r, a4i, a3i * a4r)))));
        const double t18 = t17 + t17;
        const double n7r = std::fma(c1r, a7r, std::fma(t12, a1r, std::fma(t4, a3r, std::fma(c2r, t16, std::fma(t9, a2r, std::fma(t1, a4r, std::fma(q2r, a5r, std::fma(mc1i, a7i, -std::fma(c2i, t18, std::fma(t3, a4i, std::fma(t6, a3i, std::fma(t11, a2i, std::fma(a1i, t14, q2i * a5i)))))))))))));
        const double n7i = std::fma(c1r, a7i, std::fma(c1i, a7r, std::fma(c2i, t16, std::fma(t12, a1i, std::fma(t4, a3i, std::fma(c2r, t18, std::fma(t14, a1r, std::fma(t9, a2i, std::fma(t11, a2r, std::fma(t6, a3r, std::fma(t1, a4i, std::fma(t3, a4r, std::fma(q2r, a5i, q2i * a5r)))))))))))));
        const double t19 = std::fma(2.0, std::fma(a1r, a7r, std::fma(a2r, a6r, std::fma(a3r, a5r, std::fma(t7, a7i, -std::fma(a2i, a6i, a3i * a5i))))), -std::fma(-a4r, a4r, a4i * a4i));
        const double t20 = std::fma(a1r, a7i, std::fma(a1i, a7r, std::fma(a2r, a6i, std::fma(a2i, a6r, std::fma(a3r, a5i, std::fma(a3i, a5r, a4r * a4i))))));
        const double t21 = t20 + t20;
        const double n8r = std::fma(c1r, a8r, std::fma(t19, c2r, std::fma(t12, a2r, std::fma(t4, a4r, std::fma(t16, a1r, std::fma(t9, a3r, std::fma(t1, a5r, std::fma(q2r, a6r, std::fma(mc1i, a8i, -std::fma(c2i, t21, std::fma(t3, a5i, std::fma(t6, a4i, std::fma(t11, a3i, std::fma(t14, a2i, std::fma(t18, a1i, q2i * a6i)))))))))))))));
        const double n8i = std::fma(c1r, a8i, std::fma(c1i, a8r, std::fma(c2i, t19, std::fma(t12, a2i, std::fma(t4, a4i, std::fma(c2r, t21, std::fma(t16, a1i, std::fma(t18, a1r, std::fma(t14, a2r, std::fma(t9, a3i, std::fma(t11, a3r, std::fma(t1, a5i, std::fma(t6, a4r, std::fma(t3, a5r, std::fma(q2r, a6i, q2i * a6r)))))))))))))));
        const double mag_a2 = std::fma(n1r, n1r, n1i * n1i);
        if (mag_a2 > 0.0) {
            const double mag_a = std::sqrt(mag_a2);
            const double err = std::sqrt(std::fma(n8i, n8i, n8r * n8r)) * 0.1;
            if (err / mag_a > tol || mag_a > 0.5) break;
        }
        a1r = n1r; a1i = n1i; a2r = n2r; a2i = n2i;
        a3r = n3r; a3i = n3i; a4r = n4r; a4i = n4i;
        a5r = n5r; a5i = n5i; a6r = n6r; a6i = n6i;
        a7r = n7r; a7i = n7i; a8r = n8r; a8i = n8i;
    }
    const double a[16] = {a1r, a1i, a2r, a2i, a3r, a3i, a4r, a4i, a5r, a5i, a6r, a6i, a7r, a7i, a8r, a8i};
    finish(k, ref_len, a, 16, out);
    return AP_OK;
}

// Multibrot n = 3, order 4 (math_core/high_precision.py:449-534).
int series_cubic4(const double* re, const double* im, int ref_len, double r, int ft, double kr, double ki,
           double tol, double* out) {
    double a1r = 0.0, a1i = 0.0, a2r = 0.0, a2i = 0.0;
    double a3r = 0.0, a3i = 0.0, a4r = 0.0, a4i = 0.0;
    const double cc = r;
    int k = 0;
    for (; k < ref_len; ++k) {
        const double x = re[k], y = im[k];
        const double c1r = std::fma(-3.0, std::fma(-x, x, y * y), kr);
        const double c1i = std::fma(y, x * 6.0, ki);
        const double n1r = cc + std::fma(c1r, a1r, -(c1i * a1i));
        const double n1i = std::fma(c1r, a1i, c1i * a1r);
        const double c2r = x * 3.0;
        const double q2r = std::fma(a1r, a1r, -(a1i * a1i));
        const double mc1i = -c1i;
        const double c2i = y * 3.0;
        const double q2i = a1i * (a1r + a1r);
        const double n2r = std::fma(c1r, a2r, std::fma(c2r, q2r, std::fma(mc1i, a2i, -(c2i * q2i))));
        const double n2i = std::fma(c1r, a2i, std::fma(c1i, a2r, std::fma(c2i, q2r, c2r * q2i)));
        const double t0 = std::fma(a1r, a2r, -(a1i * a2i));
        const double t1 = t0 + t0;
        const double t2 = std::fma(a1r, a2i, a1i * a2r);
        const double t3 = t2 + t2;
        const double n3r = std::fma(c1r, a3r, std::fma(c2r, t1, std::fma(q2r, a1r, std::fma(mc1i, a3i, -std::fma(c2i, t3, q2i * a1i)))));
        const double n3i = std::fma(c1r, a3i, std::fma(c1i, a3r, std::fma(c2i, t1, std::fma(c2r, t3, std::fma(q2r, a1i, q2i * a1r)))));
        const double t4 = std::fma(-std::fma(-a1r, a3r, a1i * a3i), 2.0, -std::fma(-a2r, a2r, a2i * a2i));
        const double t5 = std::fma(a1r, a3i, std::fma(a1i, a3r, a2r * a2i));
        const double t6 = t5 + t5;
        const double n4r = std::fma(c1r, a4r, std::fma(t4, c2r, std::fma(t1, a1r, std::fma(q2r, a2r, std::fma(mc1i, a4i, -std::fma(c2i, t6, std::fma(t3, a1i, q2i * a2i)))))));
        const double n4i = std::fma(c1r, a4i, std::fma(c1i, a4r, std::fma(c2i, t4, std::fma(c2r, t6, std::fma(t1, a1i, std::fma(t3, a1r, std::fma(q2r, a2i, q2i * a2r)))))));
        const double mag_a2 = std::fma(n1r, n1r, n1i * n1i);
        if (mag_a2 > 0.0) {
            const double mag_a = std::sqrt(mag_a2);
            const double err = std::sqrt(std::fma(n4r, n4r, n4i * n4i)) * 0.1;
            if (err / mag_a > tol || mag_a > 0.5) break;
        }
        a1r = n1r; a1i = n1i; a2r = n2r; a2i = n2i;
        a3r = n3r; a3i = n3i; a4r = n4r; a4i = n4i;
    }
    const double a[8] = {a1r, a1i, a2r, a2i, a3r, a3i, a4r, a4i};
    finish(k, ref_len, a, 8, out);
    return AP_OK;
}

}  // namespace

extern "C" int ap_bbsa_coeffs(const double* ref_re, const double* ref_im, int32_t ref_len,
                              double max_r, int32_t fractal_type, double tol, int32_t order,
                              int32_t gen_n, double gen_kr, double gen_ki, int32_t e_scale,
                              double* out) {
    if (!out) {
        ap::set_error("ap_bbsa_coeffs: out is null");
        return AP_E_INVALID;
    }
    std::memset(out, 0, 17 * sizeof(double));
    if (!(fractal_type == 0 || fractal_type == 2 || fractal_type == 4) || !(tol > 0.0) ||
        order <= 0 || ref_len < 2 || !(max_r > 0.0) || std::isinf(max_r) || order == 32 ||
        e_scale > 0)
        return AP_OK;
    if (!ref_re || !ref_im) {
        ap::set_error("ap_bbsa_coeffs: null orbit");
        return AP_E_INVALID;
    }
    const bool four = order == 4;
    if (fractal_type == 0 || fractal_type == 2)
        return (four ? series_quadratic4 : series_quadratic8)(ref_re, ref_im, ref_len, max_r, fractal_type,
                                                             gen_kr, gen_ki, tol, out);
    if (gen_n == 3)
        return (four ? series_cubic4 : series_cubic8)(ref_re, ref_im, ref_len, max_r, fractal_type, gen_kr,
                                                     gen_ki, tol, out);
    return AP_OK;
}
