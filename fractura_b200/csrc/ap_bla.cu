// ap_bla.cu -- chained bilinear-approximation table built on the device.
//
// Level 0 holds the one-step linearisation A_k = f'(Z_k), B_k = 1 with its
// validity radius; level d merges levels d-1 at k and k + 2^(d-1):
//   A = A2 A1,  B = A2 B1 + B2,  r^2 = min(r1^2, r2^2 / (4 |A1|^2)) <= 1/4,
// an entry being zeroed when |A|^2 or |B|^2 exceeds 1e150.
// (_jit_build_bla_table, math_core/high_precision.py:1101-1238.)  The
// reference evaluates it with a fastmath CPU kernel; the multiply-adds below
// are fused exactly where that compiled kernel fuses them, so Mandelbrot,
// Julia and Multibrot n = 2, 3 tables are byte-identical to the reference's.
// One launch per level; each level is a data-parallel map over k.
#include "ap_common.cuh"

namespace ap {

__global__ void __launch_bounds__(256) bla_level0_kernel(const double* __restrict__ re,
                                                         const double* __restrict__ im, int ref_len,
                                                         int fractal_type, double tol, int gen_n,
                                                         double kr, double ki,
                                                         double* __restrict__ T) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ref_len - 1) return;
    const double rx = re[k], ry = im[k];
    double* e = T + (size_t)k * 5;
    const double r_mag2 = fma(ry, ry, rx * rx);
    if (fractal_type == 0 || fractal_type == 2) {
        e[0] = 2.0 * rx;
        e[1] = 2.0 * ry;
        e[2] = 1.0;
        e[3] = 0.0;
        double r_sq = ((tol * tol) * 4.0) * r_mag2;
        r_sq = 0.25 < r_sq ? 0.25 : r_sq;
        if (k == 0 && r_mag2 < 1e-14) r_sq = 0.0;
        e[4] = r_sq;
        return;
    }
    // Multibrot z^n + K z + c: A = n R^(n-1) + K, radius of the quadratic bound.
    double zr = 1.0, zi = 0.0;
    for (int t = 0; t < gen_n - 1; ++t) {
        const double nr = fma(zr, rx, -(zi * ry));
        const double ni = fma(zr, ry, zi * rx);
        zr = nr;
        zi = ni;
    }
    const double ar = fma((double)gen_n, zr, kr), ai = fma((double)gen_n, zi, ki);
    e[0] = ar;
    e[1] = ai;
    e[2] = 1.0;
    e[3] = 0.0;
    const double tol_a = sqrt(fma(ai, ai, ar * ar)) * tol;
    if (!(tol_a > 0.0)) {
        e[4] = 0.0;
        return;
    }
    const double r_mag = sqrt(r_mag2);
    double r_pow;
    if (gen_n == 2) r_pow = 1.0;
    else if (gen_n == 3) r_pow = r_mag;
    else if (gen_n == 4) r_pow = r_mag2;
    else r_pow = pow(r_mag, (double)(gen_n - 2));
    const double bq = r_pow * (0.25 * (double)(gen_n * (gen_n - 1)));
    const double denom = sqrt(fma(bq, bq, tol_a)) + bq;
    double x = denom > 1e-300 ? tol_a / denom : 0.0;
    if (gen_n > 3) {
        const double x_max = pow(tol_a, 1.0 / (double)(gen_n - 1));
        if (x > x_max) x = x_max;
    }
    x = 0.5 < x ? 0.5 : x;
    double r_sq = x * x;
    if (k == 0 && r_mag2 < 1e-14) r_sq = 0.0;
    e[4] = r_sq;
}

__global__ void __launch_bounds__(256) bla_merge_kernel(double* __restrict__ T, int ref_len, int d,
                                                        int step) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ref_len - 2 * step) return;
    const size_t L = (size_t)ref_len;
    const double* e1 = T + ((size_t)(d - 1) * L + k) * 5;
    const double* e2 = T + ((size_t)(d - 1) * L + k + step) * 5;
    double* o = T + ((size_t)d * L + k) * 5;
    const double r1 = e1[4], r2 = e2[4];
    if (!(r1 > 0.0 && r2 > 0.0)) return;
    const double a1r = e1[0], a1i = e1[1], b1r = e1[2], b1i = e1[3];
    const double a2r = e2[0], a2i = e2[1], b2r = e2[2], b2i = e2[3];
    const double ar = fma(a2r, a1r, -(a2i * a1i));
    const double ai = fma(a2i, a1r, a2r * a1i);
    if (fma(ar, ar, ai * ai) > 1e150) {
        o[0] = o[1] = o[2] = o[3] = o[4] = 0.0;
        return;
    }
    const double br = fma(a2r, b1r, -(a2i * b1i)) + b2r;
    const double bi = fma(a2i, b1r, fma(a2r, b1i, b2i));
    if (fma(br, br, bi * bi) > 1e150) {
        o[0] = o[1] = o[2] = o[3] = o[4] = 0.0;
        return;
    }
    o[0] = ar;
    o[1] = ai;
    o[2] = br;
    o[3] = bi;
    const double a1_mag2 = fma(a1i, a1i, a1r * a1r);
    double rc = r1;
    if (a1_mag2 > 1e-300) {
        const double r2s = (0.25 * r2) / a1_mag2;
        rc = r1 < r2s ? r1 : r2s;
    }
    o[4] = rc <= 0.0 ? 0.0 : (rc > 0.25 ? 0.25 : rc);
}

// dc-aware merge (Zhuoran's chained BLA, fractalforums.org 2021): the second
// leap starts from dz1 = A1 dz + B1 dc, so it is valid while
// |A1| |dz| + |B1| |dc|max < r2, i.e.
//   r = max(0, min(r1, (r2 - |B1| dcmax) / |A1|)).
// Radii are stored squared as in the reference layout; the coefficients are
// merged exactly as in bla_merge_kernel.
__global__ void __launch_bounds__(256) bla_merge_dc_kernel(double* __restrict__ T, int ref_len, int d,
                                                           int step, double dc_max) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ref_len - 2 * step) return;
    const size_t L = (size_t)ref_len;
    const double* e1 = T + ((size_t)(d - 1) * L + k) * 5;
    const double* e2 = T + ((size_t)(d - 1) * L + k + step) * 5;
    double* o = T + ((size_t)d * L + k) * 5;
    const double r1s = e1[4], r2s = e2[4];
    if (!(r1s > 0.0 && r2s > 0.0)) return;
    const double a1r = e1[0], a1i = e1[1], b1r = e1[2], b1i = e1[3];
    const double a2r = e2[0], a2i = e2[1], b2r = e2[2], b2i = e2[3];
    const double ar = fma(a2r, a1r, -(a2i * a1i));
    const double ai = fma(a2i, a1r, a2r * a1i);
    const double br = fma(a2r, b1r, -(a2i * b1i)) + b2r;
    const double bi = fma(a2i, b1r, fma(a2r, b1i, b2i));
    if (fma(ar, ar, ai * ai) > 1e150 || fma(br, br, bi * bi) > 1e150) {
        o[0] = o[1] = o[2] = o[3] = o[4] = 0.0;
        return;
    }
    const double a1_mag = sqrt(fma(a1i, a1i, a1r * a1r));
    const double b1_mag = sqrt(fma(b1i, b1i, b1r * b1r));
    double r = sqrt(r1s);
    if (a1_mag > 1e-300) {
        const double r2c = (sqrt(r2s) - b1_mag * dc_max) / a1_mag;
        r = r < r2c ? r : r2c;
    }
    if (!(r > 0.0)) return;
    o[0] = ar;
    o[1] = ai;
    o[2] = br;
    o[3] = bi;
    const double rs = r * r;
    o[4] = rs < r1s ? rs : r1s;  // sqrt then square may round up by an ulp
}

// Level 0 then one merge launch per level; dc_max < 0 selects the reference merge.
static int build_bla_levels(const double* ref_re, const double* ref_im, int ref_len, int fractal_type,
                            double tol, double dc_max, int levels, int gen_n, double gen_kr,
                            double gen_ki, double* out, cudaStream_t st, const char* what) {
    const size_t bytes = sizeof(double) * 5 * (size_t)levels * (size_t)ref_len;
    if (bytes == 0) return AP_OK;
    cudaError_t e = cudaMemsetAsync(out, 0, bytes, st);
    if (e != cudaSuccess) {
        set_error("%s: memset: %s", what, cudaGetErrorString(e));
        return AP_E_CUDA;
    }
    if (!(fractal_type == 0 || fractal_type == 2 || fractal_type == 4) || ref_len < 4 || !(tol > 0.0))
        return AP_OK;
    const int blocks = (ref_len + 255) / 256;
    bla_level0_kernel<<<blocks, 256, 0, st>>>(ref_re, ref_im, ref_len, fractal_type, tol, gen_n,
                                              gen_kr, gen_ki, out);
    int rc = check_launch("bla_level0_kernel");
    int step = 1;
    for (int d = 1; d < levels && rc == AP_OK; ++d) {
        if (ref_len - 2 * step > 0) {
            if (dc_max < 0.0) {
                bla_merge_kernel<<<blocks, 256, 0, st>>>(out, ref_len, d, step);
                rc = check_launch("bla_merge_kernel");
            } else {
                bla_merge_dc_kernel<<<blocks, 256, 0, st>>>(out, ref_len, d, step, dc_max);
                rc = check_launch("bla_merge_dc_kernel");
            }
        }
        step *= 2;
    }
    return rc;
}

}  // namespace ap

extern "C" int ap_build_bla(const double* ref_re, const double* ref_im, int32_t ref_len,
                            int32_t fractal_type, double tol, int32_t levels, int32_t gen_n,
                            double gen_kr, double gen_ki, double* out, void* stream) {
    if (!ref_re || !ref_im || !out || ref_len < 0 || levels < 1 || levels > 31 || gen_n < 0 ||
        gen_n > 64) {
        ap::set_error("ap_build_bla: bad arguments");
        return AP_E_INVALID;
    }
    return ap::build_bla_levels(ref_re, ref_im, ref_len, fractal_type, tol, -1.0, levels, gen_n,
                                gen_kr, gen_ki, out, static_cast<cudaStream_t>(stream),
                                "ap_build_bla");
}

extern "C" int ap_build_bla_dc(const double* ref_re, const double* ref_im, int32_t ref_len,
                               int32_t fractal_type, double eps, double dc_max, int32_t levels,
                               int32_t gen_n, double gen_kr, double gen_ki, double* out,
                               void* stream) {
    if (!ref_re || !ref_im || !out || ref_len < 0 || levels < 1 || levels > 31 || gen_n < 0 ||
        gen_n > 64 || !(dc_max >= 0.0) || !(eps > 0.0)) {
        ap::set_error("ap_build_bla_dc: bad arguments");
        return AP_E_INVALID;
    }
    return ap::build_bla_levels(ref_re, ref_im, ref_len, fractal_type, eps, dc_max, levels, gen_n,
                                gen_kr, gen_ki, out, static_cast<cudaStream_t>(stream),
                                "ap_build_bla_dc");
}
