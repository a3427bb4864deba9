// ap_strict.cu -- Strict Metric re-evaluation of the pixels still glitched after
// rebasing, on the device.
//
// Semantics of eval_glitched_pixels_cuda_kernel / eval_glitched_pixels_hist_cuda_kernel
// (math_core/cuda_kernels.py:2450-2569) with their two deep tiers:
//   * double-double direct iteration (compute_dd_sample, :321-418) at the pixel's
//     double-double c;
//   * 34 x 32-bit sign-magnitude fixed point (compute_ml_sample, :2372-2446): limb 0
//     the integer part, 33 fraction limbs, a truncated product that keeps every
//     partial product of limbs i + j <= 33 and the high halves of i + j = 34.
//
// One thread per pixel: the fixed-point state (|z_x|, |z_y|, their squares and
// product) lives in registers, fully unrolled; each pixel's c sits in shared memory.
// Blocks are one warp so the few hundred pixels the fallback receives spread over
// as many SMs as possible: the pass is latency-bound, not throughput-bound.
#include "ap_common.cuh"
#include "ap_dd.cuh"
#include "ap_fp64.cuh"

namespace ap {
namespace {

constexpr int NL = AP_STRICT_NLIMBS;
constexpr int kStrictThreads = 32;
constexpr int kCStride = 2 * NL + 1;  // words per thread in shared memory (odd: no bank conflicts)

typedef uint32_t Limbs[NL];

// |a| + |b|; the carry out of the integer limb is dropped (ml_add_mag, :2300-2307).
__device__ __forceinline__ void ml_add_mag(const Limbs& a, const Limbs& b, Limbs& o) {
    uint64_t c = 0;
#pragma unroll
    for (int i = NL - 1; i >= 0; --i) {
        const uint64_t s = (uint64_t)a[i] + (uint64_t)b[i] + c;
        o[i] = (uint32_t)s;
        c = s >> 32;
    }
}

// |a| - |b|, wrapping below zero (ml_sub_mag, :2310-2321; callers order the operands).
__device__ __forceinline__ void ml_sub_mag(const Limbs& a, const Limbs& b, Limbs& o) {
    uint64_t borrow = 0;
#pragma unroll
    for (int i = NL - 1; i >= 0; --i) {
        const uint64_t d = (uint64_t)a[i] - (uint64_t)b[i] - borrow;
        o[i] = (uint32_t)d;
        borrow = d >> 63;
    }
}

// Sign of |a| - |b| (ml_cmp_mag): the most significant differing limb decides.
__device__ __forceinline__ int ml_cmp_mag(const Limbs& a, const Limbs& b) {
    int r = 0;
#pragma unroll
    for (int i = NL - 1; i >= 0; --i) r = a[i] > b[i] ? 1 : (a[i] < b[i] ? -1 : r);
    return r;
}

// (as, a) + (bs, b) -> o, returns the sign (ml_add_signed, :2324-2335).  o may be a.
__device__ __forceinline__ int ml_add_signed(int as, const Limbs& a, int bs, const Limbs& b, Limbs& o) {
    if (as == bs) {
        ml_add_mag(a, b, o);
        return as;
    }
    if (ml_cmp_mag(a, b) >= 0) {
        ml_sub_mag(a, b, o);
        return as;
    }
    ml_sub_mag(b, a, o);
    return bs;
}

// (as, a) - (bs, b) -> o (ml_sub_signed, :2338-2341).
__device__ __forceinline__ int ml_sub_signed(int as, const Limbs& a, int bs, const Limbs& b, Limbs& o) {
    return ml_add_signed(as, a, bs == 0 ? 1 : 0, b, o);
}

// Truncated product (ml_mul_mag, :2344-2368).  Column k (weight 2^(-32k)) sums the
// low halves of a_i b_j with i + j = k and the high halves of those with i + j = k + 1;
// the last column also takes the high halves of i + j = 34 (i >= 1).  Columns are
// carried from the least significant up; the carry out of limb 0 is dropped.  o must
// not alias a or b.
__device__ __forceinline__ void ml_mul(const Limbs& a, const Limbs& b, Limbs& o) {
    uint64_t carry = 0;
#pragma unroll
    for (int k = NL - 1; k >= 0; --k) {
        uint64_t s = carry;
#pragma unroll
        for (int i = 0; i <= k; ++i) s += (uint32_t)(a[i] * b[k - i]);
        if (k + 1 < NL) {
#pragma unroll
            for (int i = 0; i <= k + 1; ++i) s += __umulhi(a[i], b[k + 1 - i]);
        } else {
#pragma unroll
            for (int i = 1; i < NL; ++i) s += __umulhi(a[i], b[NL - i]);
        }
        o[k] = (uint32_t)s;
        carry = s >> 32;
    }
}

// ml_mul(a, a, o) with each symmetric pair of partial products formed once: every
// column sum, and so every limb, is the same integer.
__device__ __forceinline__ void ml_sqr(const Limbs& a, Limbs& o) {
    uint64_t carry = 0;
#pragma unroll
    for (int k = NL - 1; k >= 0; --k) {
        uint64_t s = carry;
        uint64_t d = 0;
#pragma unroll
        for (int i = 0; i < (k + 1) / 2; ++i) d += (uint32_t)(a[i] * a[k - i]);
        if ((k & 1) == 0) s += (uint32_t)(a[k / 2] * a[k / 2]);
        if (k + 1 < NL) {
#pragma unroll
            for (int i = 0; i < (k + 2) / 2; ++i) d += __umulhi(a[i], a[k + 1 - i]);
            if (((k + 1) & 1) == 0) s += __umulhi(a[(k + 1) / 2], a[(k + 1) / 2]);
        } else {
#pragma unroll
            for (int i = 1; i < NL / 2; ++i) d += __umulhi(a[i], a[NL - i]);
            s += __umulhi(a[NL / 2], a[NL / 2]);
        }
        s += 2 * d;
        o[k] = (uint32_t)s;
        carry = s >> 32;
    }
}

__device__ __forceinline__ void load_limbs(const uint32_t* src, Limbs& o) {
#pragma unroll
    for (int i = 0; i < NL; ++i) o[i] = src[i];
}

// compute_ml_sample (:2372-2446): z = 0, c = pixel, or z = pixel, c = Julia constant
// (types 2, 3); Burning Ship types take |z| by clearing the signs; bailout when the
// integer part of z_x^2, z_y^2 or their sum reaches 65536.
__device__ float limbs_sample(const uint32_t* s_cx, int cxs, const uint32_t* s_cy, int cys,
                              int pix_xs, int pix_ys, const uint32_t* s_px, const uint32_t* s_py,
                              int max_iter, int ft) {
    if (ft == 4) return -1.0f;
    Limbs zx, zy, zx2, zy2, zxy, t;
    int zxs = 0, zys = 0;
    if (ft == 2 || ft == 3) {
        load_limbs(s_px, zx);
        load_limbs(s_py, zy);
        zxs = pix_xs;
        zys = pix_ys;
    } else {
#pragma unroll
        for (int i = 0; i < NL; ++i) zx[i] = zy[i] = 0u;
    }
    const bool ship = ft == 1 || ft == 3;
    for (int k = 0; k < max_iter; ++k) {
        if (ship) zxs = zys = 0;
        ml_sqr(zx, zx2);
        ml_sqr(zy, zy2);
        if (zx2[0] >= 65536u || zy2[0] >= 65536u || (uint64_t)zx2[0] + (uint64_t)zy2[0] >= 65536ull) {
            const double mag2 = (double)zx2[0] + (double)zy2[0] +
                                ((double)zx2[1] + (double)zy2[1]) * 2.3283064365386963e-10;
            return escaped_sample(k, mag2, kInvLn2).s;
        }
        const int zxys = zxs == zys ? 0 : 1;
        ml_mul(zx, zy, zxy);
        ml_add_mag(zxy, zxy, zxy);
        const int subs = ml_sub_signed(0, zx2, 0, zy2, zx2);
        load_limbs(s_cx, t);
        zxs = ml_add_signed(subs, zx2, cxs, t, zx);
        load_limbs(s_cy, t);
        zys = ship ? ml_sub_signed(0, zxy, cys, t, zy) : ml_add_signed(zxys, zxy, cys, t, zy);
    }
    return -1.0f;
}

__global__ void __launch_bounds__(kStrictThreads) strict_eval_kernel(
    const ApFrameParams p, const ApFrameBuffers b, const ApStrictView v,
    const int32_t* __restrict__ coords, const int32_t* __restrict__ signs,
    const uint32_t* __restrict__ limbs, int n, int hist) {
    __shared__ uint32_t s_pix[kStrictThreads * kCStride];
    __shared__ uint32_t s_jul[2 * NL];
    for (int i = threadIdx.x; i < 2 * NL; i += blockDim.x) s_jul[i] = i < NL ? v.jx_limbs[i] : v.jy_limbs[i - NL];
    __syncthreads();
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int r = coords[2 * q], c = coords[2 * q + 1];
    if (r < 0 || r >= p.height || c < 0 || c >= p.width) return;
    float s;
    if (v.tier == AP_STRICT_DD) {
        s = dd_sample_at<AP_ARITH_REF_CUDA>(p, (double)c, (double)r).s;
    } else if (v.tier == AP_STRICT_FP64) {
        const double x = p.x_min_hi + (double)c * p.dx_hi;
        const double y = p.y_max_hi - (double)r * p.dy_hi;
        s = fp64_sample<AP_ARITH_REF_CUDA>(x, y, p).s;
    } else {
        uint32_t* mine = s_pix + threadIdx.x * kCStride;
        for (int i = 0; i < 2 * NL; ++i) mine[i] = __ldg(limbs + (size_t)q * 2 * NL + i);
        const int pxs = __ldg(signs + 2 * q), pys = __ldg(signs + 2 * q + 1);
        if (p.fractal_type == 2 || p.fractal_type == 3)
            s = limbs_sample(s_jul, v.jx_sign, s_jul + NL, v.jy_sign, pxs, pys, mine, mine + NL,
                             p.max_iter, p.fractal_type);
        else
            s = limbs_sample(mine, pxs, mine + NL, pys, 0, 0, mine, mine + NL, p.max_iter,
                             p.fractal_type);
    }
    const size_t idx = (size_t)r * p.width + c;
    b.iter_map[idx] = s;
    double cr = 0.0, cg = 0.0, cb = 0.0;
    if (s >= 0.0f) colour_of(p, b.lut, b.cdf, hist != 0, (double)s, cr, cg, cb);
    store_rgb(b.rgb, p.is_hdr, idx, cr, cg, cb);
    if (b.glitch_out) b.glitch_out[idx] = 0;
}

}  // namespace
}  // namespace ap

extern "C" int ap_strict_eval(const ApFrameParams* p, const ApFrameBuffers* b, const ApStrictView* v,
                              const int32_t* coords, const int32_t* signs, const uint32_t* limbs,
                              int32_t n, void* stream) {
    if (!p || !b || !v || !b->iter_map || !b->rgb || !b->lut || n < 0 || (n > 0 && !coords) ||
        p->width <= 0 || p->height <= 0 || p->max_iter < 0 ||
        (v->tier != AP_STRICT_DD && v->tier != AP_STRICT_LIMBS && v->tier != AP_STRICT_FP64) ||
        (v->tier == AP_STRICT_LIMBS && n > 0 && (!signs || !limbs))) {
        ap::set_error("ap_strict_eval: bad arguments");
        return AP_E_INVALID;
    }
    if (n == 0) return AP_OK;
    const int hist = (p->scheme_id == 11 && b->cdf != nullptr) ? 1 : 0;
    const int blocks = (n + ap::kStrictThreads - 1) / ap::kStrictThreads;
    ap::strict_eval_kernel<<<blocks, ap::kStrictThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        *p, *b, *v, coords, signs, limbs, n, hist);
    return ap::check_launch("strict_eval_kernel");
}
