// ap_bbsa.cu -- series-approximation start ("BBSA") coefficients, on the host.
//
// The per-pixel start of the perturbation tier (bbsa_skip, bbsa_inv_r and
// 16 coefficients in ApFrameParams) comes from a serial recurrence over the
// reference orbit: with u = dc / r, the delta after k steps is modelled as
// sum_j a_j u^j (j = 1..4 or 1..8) and the coefficients are advanced one orbit
// step at a time until the truncation estimate exceeds the tolerance or the
// linear term exceeds 1/2.  This is _jit_compute_bbsa_coeffs
// (math_core/high_precision.py:50-535) for Mandelbrot, Julia and Multibrot
// n = 3; every other case returns skip 0.  One dependent chain of complex
// products per orbit step, computed once per reference orbit: it runs on the
// host, beside the orbit it reads, and takes microseconds per thousand steps.
#include <cmath>
#include <cstring>

#include "ap_common.cuh"

namespace {

struct C2 {
    double r, i;
};

inline C2 mul(C2 a, C2 b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
inline C2 add(C2 a, C2 b) { return {a.r + b.r, a.i + b.i}; }
inline C2 twice(C2 a) { return {2.0 * a.r, 2.0 * a.i}; }
inline double mag(C2 a) { return std::sqrt(a.r * a.r + a.i * a.i); }
inline bool bad(double x) { return std::isnan(x) || std::isinf(x); }

// Sum of a[p] * a[q] over p < q, p + q = n (indices from 1), left to right.
inline C2 cross(const C2* a, int n) {
    C2 s{0.0, 0.0};
    bool first = true;
    for (int p = 1; 2 * p < n; ++p) {
        const C2 t = mul(a[p], a[n - p]);
        s = first ? t : add(s, t);
        first = false;
    }
    return s;
}

// q_n = sum over p + q = n of a_p a_q: 2 * cross (+ a_{n/2}^2 for even n).
inline C2 square_coeff(const C2* a, int n) {
    if (n == 2) return mul(a[1], a[1]);
    const C2 c = twice(cross(a, n));
    if (n % 2 == 0) {
        const C2 s = mul(a[n / 2], a[n / 2]);
        return add(c, s);
    }
    return c;
}

// Mandelbrot / Julia: a' = 2 Z a + (a^2 terms) + c_const [j = 1].
int series_quadratic(const double* re, const double* im, int ref_len, double r, int ft, int order,
                     double tol, double* out) {
    C2 a[10] = {}, best[10] = {};
    if (ft == 2) a[1] = {r, 0.0};
    const C2 c_const{ft == 0 ? r : 0.0, 0.0};
    for (int j = 1; j <= order; ++j) best[j] = a[j];
    int skip = 0;
    for (int k = 0; k < ref_len; ++k) {
        const C2 c1{2.0 * re[k], 2.0 * im[k]};
        C2 q[10];
        for (int n = 2; n <= order + 1; ++n) q[n] = square_coeff(a, n);
        C2 nx[10];
        nx[1] = add(mul(c1, a[1]), c_const);
        for (int j = 2; j <= order; ++j) nx[j] = add(mul(c1, a[j]), q[j]);
        const double lin = mag(nx[1]), top = mag(nx[order]);
        if (bad(lin) || bad(top)) break;
        const double err = mag(q[order + 1]) + top * 0.1;
        if (lin > 0.0 && (err / lin > tol || lin > 0.5)) break;
        for (int j = 1; j <= order; ++j) a[j] = best[j] = nx[j];
        skip = k + 1;
    }
    const int cap = ref_len - 2 > 0 ? ref_len - 2 : 0;
    out[0] = (double)(skip < cap ? skip : cap);
    for (int j = 1; j <= order; ++j) {
        out[2 * j - 1] = best[j].r;
        out[2 * j] = best[j].i;
    }
    return AP_OK;
}

// Multibrot n = 3 (z^3 + K z + c): a' = (3 Z^2 + K) a + 3 Z (a^2 terms) + (a^3 terms) + c_const.
int series_cubic(const double* re, const double* im, int ref_len, double r, int order, double kr,
                 double ki, double tol, double* out) {
    C2 a[10] = {}, best[10] = {};
    const C2 c_const{r, 0.0};
    int skip = 0;
    for (int k = 0; k < ref_len; ++k) {
        const C2 z{re[k], im[k]};
        const C2 z2 = mul(z, z);
        const C2 c1{3.0 * z2.r + kr, 3.0 * z2.i + ki};
        const C2 c2{3.0 * z.r, 3.0 * z.i};
        C2 q[10];
        for (int n = 2; n <= order; ++n) q[n] = square_coeff(a, n);
        C2 w[10];  // w_n = sum_{m=2}^{n-1} q_m a_{n-m}: the cubic terms
        for (int n = 3; n <= order; ++n) {
            C2 s = mul(q[2], a[n - 2]);
            for (int m = 3; m <= n - 1; ++m) s = add(s, mul(q[m], a[n - m]));
            w[n] = s;
        }
        C2 nx[10];
        nx[1] = add(mul(c1, a[1]), c_const);
        nx[2] = add(mul(c1, a[2]), mul(c2, q[2]));
        for (int j = 3; j <= order; ++j) nx[j] = add(add(mul(c1, a[j]), mul(c2, q[j])), w[j]);
        const double lin = mag(nx[1]), top = mag(nx[order]);
        if (bad(lin) || bad(top)) break;
        const double err = top * 0.1;
        if (lin > 0.0 && (err / lin > tol || lin > 0.5)) break;
        for (int j = 1; j <= order; ++j) a[j] = best[j] = nx[j];
        skip = k + 1;
    }
    const int cap = ref_len - 2 > 0 ? ref_len - 2 : 0;
    out[0] = (double)(skip < cap ? skip : cap);
    for (int j = 1; j <= order; ++j) {
        out[2 * j - 1] = best[j].r;
        out[2 * j] = best[j].i;
    }
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
    const int n = order == 4 ? 4 : 8;
    if (fractal_type == 0 || fractal_type == 2)
        return series_quadratic(ref_re, ref_im, ref_len, max_r, fractal_type, n, tol, out);
    if (gen_n == 3) return series_cubic(ref_re, ref_im, ref_len, max_r, n, gen_kr, gen_ki, tol, out);
    return AP_OK;
}
