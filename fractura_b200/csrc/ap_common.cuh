// ap_common.cuh -- shared device helpers of the B200 escape-time engine.
//
// Compiled with -fmad=false: no multiply-add is fused unless it is written
// with fma() below, so the arithmetic in the source is the arithmetic that
// runs (the escape step of a boundary pixel depends on it).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "apeiron_b200.h"

namespace ap {

// config.py:25-26
constexpr double kInvLn2 = 1.4426950408889634;
constexpr double kLnBailoutLog = 1.7129177284488854;
constexpr double kBailout = 65536.0;

// Error reporting of the C ABI (thread-local message).
void set_error(const char* fmt, ...);
int check_launch(const char* what);

// Coarse-pass perturbation kernel on packed inputs (ap_perturb_fast.cu);
// AP_E_UNSUPPORTED when the pass is not one it serves.
int launch_perturb_fast(const ApFrameParams& p, const ApFrameBuffers& b, cudaStream_t st);
int launch_perturb_fast_rows(const ApFrameParams& p, const ApFrameBuffers& b, int row0, int rows,
                             cudaStream_t st);

// FP32-mantissa FloatExp tier (ap_fe32.cu).
int launch_fe32(const ApFrameParams& p, const ApFrameBuffers& b, cudaStream_t st);

struct SampleOut {
    float s;      // float32 smooth value (reference storage type), -1 interior
    double s64;   // float64 smooth value
    int k;        // escape step, -1 = never escaped, -2 = cardioid/bulb skip
    int glitch;
    int iters;    // iterations stepped one at a time (work accounting)
    int leaps;    // BLA leaps taken
    int iters2;   // perturbation stage-2 direct steps
};

__device__ __forceinline__ SampleOut interior_sample() {
    SampleOut o;
    o.s = -1.0f;
    o.s64 = -1.0;
    o.k = -1;
    o.glitch = 0;
    o.iters = 0;
    o.leaps = 0;
    o.iters2 = 0;
    return o;
}

// Never escaped within max_iter iterations.
__device__ __forceinline__ SampleOut interior_after(int max_iter) {
    SampleOut o = interior_sample();
    o.iters = max_iter;
    return o;
}

// Pixel removed by the Mandelbrot cardioid/bulb test: interior, zero iterations.
__device__ __forceinline__ SampleOut skipped_sample() {
    SampleOut o = interior_sample();
    o.k = -2;
    return o;
}

// f32(k+1) - f32(nu), nu = (ln(ln|z|^2 / 2) - ln(8 ln 2)) / ln n
// (math_core/cuda_kernels.py:280; math_core/cpu_kernels.py:249).
__device__ __forceinline__ SampleOut escaped_sample(int k, double mag2, double inv_ln) {
    SampleOut o;
    const double log_mag = log(mag2);
    o.k = k;
    o.glitch = 0;
    o.iters = k;
    o.leaps = 0;
    o.iters2 = 0;
    if (log_mag > 1.0) {
        const double nu = (log(0.5 * log_mag) - kLnBailoutLog) * inv_ln;
        o.s = __fsub_rn((float)((double)k + 1.0), (float)nu);
        o.s64 = ((double)k + 1.0) - nu;
    } else {
        o.s = (float)k;
        o.s64 = (double)k;
    }
    return o;
}

// 1/ln(n) rounded through float32 for Multibrot, else 1/ln 2.
__host__ __device__ __forceinline__ double inv_ln_for(int fractal_type, int gen_n) {
    if (fractal_type == 4 && gen_n > 1) return (double)(float)(1.0 / log((double)gen_n));
    return kInvLn2;
}

// ---------------------------------------------------------------- colouring
// Transfer functions of math_core/cuda_kernels.py:157-259, evaluated in
// float64 on the float32 smooth value.

__device__ __forceinline__ double py_mod(double x, double m) {
    double r = fmod(x, m);
    if (r != 0.0) {
        if ((r < 0.0) != (m < 0.0)) r += m;
    } else {
        r = copysign(0.0, m);
    }
    return r;
}

__device__ __forceinline__ double tri_wave(double phase) {
    return 1.0 - fabs((phase < 0.0 ? phase + 2.0 : phase) - 1.0);
}

// sqrt of the smooth value: the CPU reference holds it as float32 and Numba
// evaluates math.sqrt(float32) in float32; the CUDA reference holds float64.
__device__ __forceinline__ double sqrt_s(double s, bool f32) {
    return f32 ? (double)__fsqrt_rn((float)s) : sqrt(s);
}

static __device__ __noinline__ double palette_norm(double s, int scheme, double off, double density,
                                                   double contrast, bool f32) {
    const double dens = density <= 0.0 ? 1.0 : density;
    const double cont = contrast <= 0.0 ? 1.0 : contrast;
    const double kTwoPi = 6.28318530718;
    switch (scheme) {
    case 1:
        return tri_wave(py_mod(log(s * cont + 1.0) * (0.45 * dens) + off * 2.0, 2.0));
    case 2: {
        const double tri = tri_wave(py_mod(sqrt_s(s, f32) * (0.125 * dens) + off * 2.0, 2.0));
        const double k = 4.0 * cont;
        const double td = tanh(0.5 * k);
        const double scale = fabs(td) > 1e-7 ? 0.5 / td : 0.5186574;
        return 0.5 + tanh((tri - 0.5) * k) * scale;
    }
    case 3: {
        const double tri = tri_wave(py_mod(sqrt_s(s, f32) * (0.125 * dens) + off * 2.0, 2.0));
        const double k = 3.0 * cont;
        const double ed = exp(k) - 1.0;
        const double scale = fabs(ed) > 1e-7 ? 1.0 / ed : 0.0523957;
        return (exp(k * tri) - 1.0) * scale;
    }
    case 4: {
        const double tri = tri_wave(py_mod(sqrt_s(s, f32) * (0.5 * dens) + off * 2.0, 2.0));
        return cont != 1.0 ? pow(tri, cont) : tri;
    }
    case 5: {
        const double ang = s * (0.05 * dens) + off * kTwoPi;
        const double ratio = 1.61803398875 * cont;
        return 0.5 + 0.25 * (sin(ang) + sin(ang * ratio));
    }
    case 6: {
        const double ang = s * (0.08 * dens) + off * kTwoPi;
        const double val = 0.5 * (1.0 - cos(ang));
        return cont != 1.0 ? pow(val, cont) : val;
    }
    case 7: {
        const double ph = s * (0.05 * dens) + off * kTwoPi;
        const double b = 0.5 * cont;
        const double wave = sin(ph) + b * sin(ph * 2.0 + 1.2) + (b * b) * sin(ph * 4.0 + 2.4) +
                            (b * b * b) * sin(ph * 8.0 + 3.6);
        const double ns = 1.0 + b + b * b + b * b * b;
        const double scale = ns > 1e-7 ? 0.5 / ns : 0.26666666666666666;
        return 0.5 + scale * wave;
    }
    case 8: {
        double tri = tri_wave(py_mod(sqrt_s(s, f32) * (0.1 * dens) + off * 2.0, 2.0));
        if (cont != 1.0) tri = pow(tri, cont);
        const double t2 = tri * tri;
        return t2 * tri * (tri * (tri * 6.0 - 15.0) + 10.0);
    }
    case 9: {
        const double ang = s * (0.04 * dens) + (s * s) * (0.00008 * dens * cont) + off * kTwoPi;
        return 0.5 + 0.5 * sin(ang);
    }
    case 10: {
        const double raw = py_mod(1.0 - exp(-0.06 * cont * sqrt(s * dens)) + off, 1.0);
        return raw >= 0.0 ? raw : raw + 1.0;
    }
    default: {  // scheme 0 and every id above 10
        const double tri = tri_wave(py_mod(sqrt_s(s, f32) * (0.125 * dens) + off * 2.0, 2.0));
        return cont != 1.0 ? pow(tri, cont) : tri;
    }
    }
}

// Histogram-equalised transfer (math_core/cuda_kernels.py:237-259).
__device__ __forceinline__ double cdf_norm(double s, int max_iter, const float* __restrict__ cdf,
                                           int num_bins, double off, double density,
                                           double contrast) {
    if (s < 0.0) return -1.0;
    const double inv_max = 1.0 / fmax(1.0, (double)max_iter);
    const double pos = (s * inv_max) * (double)(num_bins - 1);
    const int k = (int)pos;
    double c;
    if (k >= num_bins - 1) {
        c = (double)__ldg(cdf + num_bins - 1);
    } else if (k < 0) {
        c = (double)__ldg(cdf);
    } else {
        const double frac = pos - (double)k;
        const float c0 = __ldg(cdf + k), c1 = __ldg(cdf + k + 1);
        c = (double)c0 + frac * (double)__fsub_rn(c1, c0);
    }
    if (contrast != 1.0 && contrast > 0.0) c = pow(c, contrast);
    const double dens = density <= 0.0 ? 1.0 : density;
    return tri_wave(py_mod(c * (2.0 * dens) + off * 2.0, 2.0));
}

// 2048-entry LUT lerp (math_core/cuda_kernels.py:157-168).
__device__ __forceinline__ void lut_lerp(const float* __restrict__ lut, double norm, double& r,
                                         double& g, double& b) {
    const double n = norm < 0.0 ? 0.0 : (norm > 1.0 ? 1.0 : norm);
    const double pos = n * 2047.0;
    const int i0 = (int)pos;
    const int i1 = i0 >= 2047 ? 2047 : i0 + 1;
    const double frac = pos - (double)i0;
    const double inv = 1.0 - frac;
    r = (double)__ldg(lut + i0 * 3 + 0) * inv + (double)__ldg(lut + i1 * 3 + 0) * frac;
    g = (double)__ldg(lut + i0 * 3 + 1) * inv + (double)__ldg(lut + i1 * 3 + 1) * frac;
    b = (double)__ldg(lut + i0 * 3 + 2) * inv + (double)__ldg(lut + i1 * 3 + 2) * frac;
}

__device__ __forceinline__ void store_rgb(void* rgb, int is_hdr, size_t idx, double r, double g,
                                          double b) {
    if (is_hdr) {
        uint16_t* o = static_cast<uint16_t*>(rgb) + idx * 3;
        o[0] = (uint16_t)(long long)(r + 0.5);
        o[1] = (uint16_t)(long long)(g + 0.5);
        o[2] = (uint16_t)(long long)(b + 0.5);
    } else {
        uint8_t* o = static_cast<uint8_t*>(rgb) + idx * 3;
        o[0] = (uint8_t)(long long)(r + 0.5);
        o[1] = (uint8_t)(long long)(g + 0.5);
        o[2] = (uint8_t)(long long)(b + 0.5);
    }
}

// Colour of one smooth value under the frame's transfer function.
__device__ __forceinline__ void colour_of(const ApFrameParams& p, const float* __restrict__ lut,
                                          const float* __restrict__ cdf, bool hist, double s,
                                          double& r, double& g, double& b) {
    const double norm = hist ? cdf_norm(s, p.max_iter, cdf, p.num_bins, p.palette_offset,
                                        p.color_density, p.color_contrast)
                             : palette_norm(s, p.scheme_id, p.palette_offset, p.color_density,
                                            p.color_contrast, p.arith == AP_ARITH_REF_CPU);
    lut_lerp(lut, norm, r, g, b);
}

}  // namespace ap
