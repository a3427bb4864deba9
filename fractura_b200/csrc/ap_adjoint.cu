// ap_adjoint.cu -- derivatives of the smooth escape value (FP64 direct tier).
//
// For a view (centre cx + i cy, width w, W x H pixels) and a formula with a
// complex parameter P (Julia: z0 = pixel, z' = z^2 + P; Multibrot:
// z' = z^n + P z + pixel; Mandelbrot: z' = z^2 + pixel, no parameter), the
// smooth value of an escaping pixel is
//   s = (K + 1) - (ln(0.5 ln m) - LN_BAILOUT_LOG) / ln n,   m = |z_K|^2 > 65536,
// so ds/dz_K = -(2 / ln n) z_K / (m ln m) (zero where ln m <= 1 or the pixel stays
// bounded or is skipped by the cardioid/bulb test).  The five real parameters
// theta = (cx, cy, ln w, Re P, Im P) enter through the pixel's position
// (x = cx - w/2 + i w/(W-1), y = cy + h/2 - j h/(H-1), h = w H / W) and P.
//
//   ap_smooth_forward: s, K and checkpoints z_0, z_C, z_2C, ... (C = ckpt_every);
//   ap_smooth_adjoint: per pixel, for the upstream gradient g = dL/ds, sweeps the
//     orbit backwards one checkpoint segment at a time, recomputing the segment's
//     z from its checkpoint (first every 16th z, then each 16-step sub-segment into
//     shared memory; no orbit is stored), and accumulates dL/dtheta; one row of sums
//     per warp of 8 x 4 pixels (deterministic, summed by the caller);
//   ap_smooth_tangent: forward mode (one tangent per parameter carried beside z),
//     per-pixel ds/dtheta, the independent check of the adjoint.
// Holomorphic steps make both sweeps complex multiplications: the adjoint
// multiplies by conj(f'(z_k)), the tangent by f'(z_k).
#include "ap_common.cuh"

namespace ap {

constexpr int kMaxSegment = 1024;
// The adjoint replays a checkpoint segment twice: once keeping z every kSub steps (local
// memory, kMaxSubs values), then, sub-segment by sub-segment from the last, to hold that
// sub-segment's z in shared memory for the reverse sweep.  No orbit reaches global memory.
constexpr int kSub = 16;
constexpr int kMaxSubs = kMaxSegment / kSub;

struct C2d {
    double r, i;
};
__device__ __forceinline__ C2d cmul2(C2d a, C2d b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
__device__ __forceinline__ C2d cadd2(C2d a, C2d b) { return {a.r + b.r, a.i + b.i}; }

// z' = f(z) and f'(z) for the three formulas.
__device__ __forceinline__ void step_f(const ApGradView& v, C2d z, C2d c, C2d& zn, C2d& dfdz) {
    if (v.fractal_type == 4 && v.gen_n == 3) {
        // the generic loop's values (z^2 = z z, z^3 = z^2 z, the same sums) without its
        // first product by 1: two fewer dependent multiplies per step
        const C2d z2 = cmul2(z, z);
        const C2d P = {v.pr, v.pi};
        zn = cadd2(cadd2(cmul2(z2, z), cmul2(P, z)), c);
        dfdz = cadd2({3.0 * z2.r, 3.0 * z2.i}, P);
    } else if (v.fractal_type == 4) {
        C2d zp = {1.0, 0.0};  // z^(n-1)
        for (int t = 0; t < v.gen_n - 1; ++t) zp = cmul2(zp, z);
        const C2d P = {v.pr, v.pi};
        zn = cadd2(cadd2(cmul2(zp, z), cmul2(P, z)), c);
        dfdz = cadd2({(double)v.gen_n * zp.r, (double)v.gen_n * zp.i}, P);
    } else {
        zn = cadd2(cmul2(z, z), c);
        dfdz = {2.0 * z.r, 2.0 * z.i};
    }
}

__device__ __forceinline__ void pixel_setup(const ApGradView& v, int i, int j, C2d& z0, C2d& c,
                                            double& dpx_dw, double& dpy_dw, bool& skip) {
    const double h = v.w * (double)v.height / (double)v.width;
    const double dx = v.w / (double)max(1, v.width - 1), dy = h / (double)max(1, v.height - 1);
    const double x = (v.cx - 0.5 * v.w) + (double)i * dx;
    const double y = (v.cy + 0.5 * h) - (double)j * dy;
    dpx_dw = -0.5 + (double)i / (double)max(1, v.width - 1);
    dpy_dw = ((double)v.height / (double)v.width) * (0.5 - (double)j / (double)max(1, v.height - 1));
    skip = false;
    if (v.fractal_type == 2) {
        z0 = {x, y};
        c = {v.pr, v.pi};
    } else {
        z0 = {0.0, 0.0};
        c = {x, y};
        if (v.fractal_type == 0) {  // main cardioid and period-2 bulb: interior
            const double xm = x - 0.25, y2 = y * y, q = xm * xm + y2;
            skip = (q * (q + xm) <= 0.25 * y2) || ((x + 1.0) * (x + 1.0) + y2 <= 0.0625);
        }
    }
}

__device__ __forceinline__ double inv_ln_of(const ApGradView& v) {
    return (v.fractal_type == 4 && v.gen_n > 1) ? 1.0 / log((double)v.gen_n) : kInvLn2;
}

// Blocks of 8 x 8 pixels (two warps of 8 x 4): a block lives as long as its slowest
// pixel, so small blocks let the SMs refill as blocks finish, and the grid of a 512 x 512
// view (4096 blocks) is resident at once (32 blocks of 64 threads per SM: 4736).
__global__ void __launch_bounds__(64) smooth_forward_kernel(const ApGradView v, double* __restrict__ s64,
                                                            int32_t* __restrict__ kmap,
                                                            double2* __restrict__ ckpt, int n_ck) {
    const int i = blockIdx.x * 8 + (threadIdx.x & 7);
    const int j = blockIdx.y * 8 + (threadIdx.x >> 3);
    if (i >= v.width || j >= v.height) return;
    const size_t idx = (size_t)j * v.width + i;
    C2d z, c, d;
    double a, b;
    bool skip;
    pixel_setup(v, i, j, z, c, a, b, skip);
    double s = -1.0;
    int K = -1;
    if (!skip) {
        int until_ck = 0, slot = 0;  // steps to the next checkpoint, and its slot
        for (int k = 0; k < v.max_iter; ++k) {
            if (until_ck == 0) {
                if (ckpt && slot < n_ck) ckpt[idx * n_ck + slot] = make_double2(z.r, z.i);
                ++slot;
                until_ck = v.ckpt_every;
            }
            --until_ck;
            const double m = z.r * z.r + z.i * z.i;
            if (m > kBailout) {
                const double lm = log(m);
                s = lm > 1.0 ? ((double)k + 1.0) - (log(0.5 * lm) - kLnBailoutLog) * inv_ln_of(v)
                             : (double)k;
                K = k;
                break;
            }
            step_f(v, z, c, z, d);
        }
    }
    s64[idx] = s;
    if (kmap) kmap[idx] = skip ? -2 : K;
}

// ds/dz_K as a real 2-vector; zero when the smooth term is constant.
__device__ __forceinline__ C2d ds_dzK(const ApGradView& v, C2d zK) {
    const double m = zK.r * zK.r + zK.i * zK.i, lm = log(m);
    if (!(lm > 1.0)) return {0.0, 0.0};
    const double f = -2.0 * inv_ln_of(v) / (m * lm);
    return {f * zK.r, f * zK.i};
}

// Each warp takes 8 x 4 pixels and writes its own row of sums (shuffles, no block
// barrier); a block of kAdjWarps warps holds its shared sub-segment buffer until its
// slowest pixel is done, so small blocks keep the SMs filling up behind long-lived pixels.
#ifndef AP_ADJ_WARPS
#define AP_ADJ_WARPS 4
#endif
constexpr int kAdjWarps = AP_ADJ_WARPS;

__global__ void __launch_bounds__(32 * kAdjWarps) smooth_adjoint_kernel(const ApGradView v,
                                                                        const double* __restrict__ grad_s,
                                                                        const int32_t* __restrict__ kmap,
                                                                        const double2* __restrict__ ckpt,
                                                                        int n_ck, double* __restrict__ pix_grads,
                                                                        double* __restrict__ block_sums,
                                                                        int n_tiles) {
    __shared__ double2 buf[kSub][32 * kAdjWarps];  // one sub-segment of z per thread (8 KiB per warp)
    const int tile = blockIdx.x * kAdjWarps + (threadIdx.x >> 5);
    if (tile >= n_tiles) return;  // whole warps only: the shuffles below stay full
    const int lane = threadIdx.x & 31;
    const int tpr = (v.width + 7) / 8;
    const int bx = tile % tpr, by = tile / tpr;
    const int i = bx * 8 + (lane & 7);
    const int j = by * 4 + (lane >> 3);
    double g[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // cx, cy, ln w, Re P, Im P
    if (i < v.width && j < v.height) {
        const size_t idx = (size_t)j * v.width + i;
        const int K = kmap[idx];
        const double gs = grad_s[idx];
        if (K > 0 && gs != 0.0) {
            C2d z0, c;
            double dpx_dw, dpy_dw;
            bool skip;
            pixel_setup(v, i, j, z0, c, dpx_dw, dpy_dw, skip);
            double2 sub[kMaxSubs];  // this segment's sub-checkpoints (local memory, 1 KiB)
            const int C = v.ckpt_every;
            C2d G = {0.0, 0.0};  // dL/dz_{k+1} during the sweep
            C2d gc = {0.0, 0.0}, gp = {0.0, 0.0};
            bool first = true;
            for (int sg = K / C; sg >= 0; --sg) {
                const int k0 = sg * C;
                const int k1 = min(K, k0 + C);  // this segment's steps z_k -> z_{k+1}, k in [k0, k1)
                const double2 st = ckpt[idx * n_ck + sg];
                C2d z = {st.x, st.y}, d;
                for (int k = k0; k < k1; ++k) {  // pass 1: z every kSub steps
                    if (((k - k0) & (kSub - 1)) == 0) sub[(k - k0) / kSub] = make_double2(z.r, z.i);
                    step_f(v, z, c, z, d);
                }
                if (first) {  // the last segment ends at k1 = K: z is z_K
                    const C2d dz = ds_dzK(v, z);
                    G = {gs * dz.r, gs * dz.i};
                    first = false;
                }
                for (int s0 = k0 + ((k1 - k0 - 1) / kSub) * kSub; s0 >= k0 && k1 > k0; s0 -= kSub) {
                  const int s1 = min(k1, s0 + kSub);
                  {  // pass 2: this sub-segment's inputs z_s0 .. z_(s1-1) into shared memory
                    const double2 w0 = sub[(s0 - k0) / kSub];
                    C2d w = {w0.x, w0.y}, dw;
                    for (int k = s0; k < s1; ++k) {
                        buf[k - s0][threadIdx.x] = make_double2(w.r, w.i);
                        step_f(v, w, c, w, dw);
                    }
                  }
                  for (int k = s1 - 1; k >= s0; --k) {
                    const double2 bk = buf[k - s0][threadIdx.x];
                    const C2d zk = {bk.x, bk.y};
                    // parameter terms of z_{k+1} = f(z_k)
                    if (v.fractal_type == 2) {
                        gp = cadd2(gp, G);  // dz'/dP = 1
                    } else {
                        gc = cadd2(gc, G);  // dz'/dc = 1
                        if (v.fractal_type == 4) {  // dz'/d(Re P) = z_k, dz'/d(Im P) = i z_k
                            gp.r += G.r * zk.r + G.i * zk.i;
                            gp.i += -G.r * zk.i + G.i * zk.r;
                        }
                    }
                    C2d zn, dfdz;
                    step_f(v, zk, c, zn, dfdz);
                    G = cmul2(G, {dfdz.r, -dfdz.i});  // G_k = G_{k+1} conj(f'(z_k))
                  }
                }
            }
            if (v.fractal_type == 2) gc = G;  // the pixel is z_0
            g[0] = gc.r;
            g[1] = gc.i;
            g[2] = v.w * (gc.r * dpx_dw + gc.i * dpy_dw);
            g[3] = gp.r;
            g[4] = gp.i;
        }
        if (pix_grads) {
            for (int q = 0; q < 5; ++q) pix_grads[idx * 5 + q] = g[q];
        }
    }
    // the warp's sums, by halves (a fixed order: the result does not depend on timing)
    for (int o = 16; o > 0; o >>= 1)
        for (int q = 0; q < 5; ++q) g[q] += __shfl_down_sync(0xffffffffu, g[q], o);
    if (lane == 0)
        for (int q = 0; q < 5; ++q) block_sums[(size_t)tile * 5 + q] = g[q];
}

__global__ void __launch_bounds__(256) smooth_tangent_kernel(const ApGradView v, double* __restrict__ ds) {
    const int i = blockIdx.x * 16 + (threadIdx.x & 15);
    const int j = blockIdx.y * 16 + (threadIdx.x >> 4);
    if (i >= v.width || j >= v.height) return;
    const size_t idx = (size_t)j * v.width + i;
    C2d z, c;
    double dpx_dw, dpy_dw;
    bool skip;
    pixel_setup(v, i, j, z, c, dpx_dw, dpy_dw, skip);
    // tangents dz/dtheta for theta = cx, cy, ln w, Re P, Im P
    C2d t[5];
    for (int q = 0; q < 5; ++q) t[q] = {0.0, 0.0};
    const C2d dpix[3] = {{1.0, 0.0}, {0.0, 1.0}, {v.w * dpx_dw, v.w * dpy_dw}};
    if (v.fractal_type == 2)
        for (int q = 0; q < 3; ++q) t[q] = dpix[q];
    double out[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (!skip) {
        for (int k = 0; k < v.max_iter; ++k) {
            const double m = z.r * z.r + z.i * z.i;
            if (m > kBailout) {
                if (k > 0) {
                    const C2d g = ds_dzK(v, z);
                    for (int q = 0; q < 5; ++q) out[q] = g.r * t[q].r + g.i * t[q].i;
                }
                break;
            }
            C2d zn, dfdz;
            step_f(v, z, c, zn, dfdz);
            for (int q = 0; q < 5; ++q) t[q] = cmul2(dfdz, t[q]);
            if (v.fractal_type == 2) {
                t[3].r += 1.0;  // dz'/d(Re P) = 1
                t[4].i += 1.0;  // dz'/d(Im P) = i
            } else {
                for (int q = 0; q < 3; ++q) t[q] = cadd2(t[q], dpix[q]);  // dz'/dc
                if (v.fractal_type == 4) {
                    t[3] = cadd2(t[3], z);                // dz'/d(Re P) = z
                    t[4] = cadd2(t[4], {-z.i, z.r});      // dz'/d(Im P) = i z
                }
            }
            z = zn;
        }
    }
    for (int q = 0; q < 5; ++q) ds[idx * 5 + q] = out[q];
}

static int check_view(const ApGradView* v, const char* what) {
    if (!v || v->width < 1 || v->height < 1 || v->max_iter < 0 || v->ckpt_every < 1 ||
        v->ckpt_every > kMaxSegment || !(v->fractal_type == 0 || v->fractal_type == 2 || v->fractal_type == 4) ||
        (v->fractal_type == 4 && (v->gen_n < 2 || v->gen_n > 64)) || !(v->w > 0.0)) {
        set_error("%s: bad view (types 0, 2, 4; 1 <= ckpt_every <= %d)", what, kMaxSegment);
        return AP_E_INVALID;
    }
    return AP_OK;
}

}  // namespace ap

extern "C" int ap_smooth_forward(const ApGradView* v, double* s64, int32_t* kmap, double* ckpt,
                                 int32_t n_ck, void* stream) {
    int rc = ap::check_view(v, "ap_smooth_forward");
    if (rc != AP_OK) return rc;
    if (!s64 || (ckpt && n_ck < (v->max_iter + v->ckpt_every - 1) / v->ckpt_every + 1)) {
        ap::set_error("ap_smooth_forward: s64 required; ckpt needs ceil(max_iter / ckpt_every) + 1 slots");
        return AP_E_INVALID;
    }
    dim3 grid((v->width + 7) / 8, (v->height + 7) / 8);
    ap::smooth_forward_kernel<<<grid, 64, 0, static_cast<cudaStream_t>(stream)>>>(
        *v, s64, kmap, reinterpret_cast<double2*>(ckpt), n_ck);
    return ap::check_launch("smooth_forward_kernel");
}

extern "C" int32_t ap_smooth_adjoint_blocks(int32_t width, int32_t height) {
    return ((width + 7) / 8) * ((height + 3) / 4);
}

extern "C" int ap_smooth_adjoint(const ApGradView* v, const double* grad_s, const int32_t* kmap,
                                 const double* ckpt, int32_t n_ck, double* pix_grads,
                                 double* block_sums, void* stream) {
    int rc = ap::check_view(v, "ap_smooth_adjoint");
    if (rc != AP_OK) return rc;
    if (!grad_s || !kmap || !ckpt || !block_sums ||
        n_ck < (v->max_iter + v->ckpt_every - 1) / v->ckpt_every + 1) {
        ap::set_error("ap_smooth_adjoint: grad_s, kmap, ckpt (from ap_smooth_forward) and block_sums "
                      "are required");
        return AP_E_INVALID;
    }
    const int blocks = ap_smooth_adjoint_blocks(v->width, v->height);
    ap::smooth_adjoint_kernel<<<(blocks + ap::kAdjWarps - 1) / ap::kAdjWarps, 32 * ap::kAdjWarps, 0,
                                static_cast<cudaStream_t>(stream)>>>(
        *v, grad_s, kmap, reinterpret_cast<const double2*>(ckpt), n_ck, pix_grads, block_sums, blocks);
    return ap::check_launch("smooth_adjoint_kernel");
}

extern "C" int ap_smooth_tangent(const ApGradView* v, double* ds, void* stream) {
    int rc = ap::check_view(v, "ap_smooth_tangent");
    if (rc != AP_OK) return rc;
    if (!ds) {
        ap::set_error("ap_smooth_tangent: ds required");
        return AP_E_INVALID;
    }
    dim3 grid((v->width + 15) / 16, (v->height + 15) / 16);
    ap::smooth_tangent_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(*v, ds);
    return ap::check_launch("smooth_tangent_kernel");
}
