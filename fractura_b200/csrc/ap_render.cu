// ap_render.cu -- unified render passes (coarse / full supersample / edge
// supersample) for every precision tier, behind ap_render_pass and
// ap_resolve_hist_pass.
//
// One thread per output pixel on 16x16 tiles: a warp covers two 16-pixel
// rows, so neighbouring pixels with similar escape steps share a warp.
#include <cstdio>

#include "ap_common.cuh"
#include "ap_fp64.cuh"
#include "ap_tiers.cuh"

namespace ap {

// Blocks of kTile x kTile pixels (warps of 8 x 4).  A block lives as long as its slowest
// pixel; small blocks let an SM refill as each one ends, instead of holding 8 warps for the
// one long-lived pixel of a 16 x 16 tile.
constexpr int kTile = 8;

template <int TIER, int ARITH>
__device__ __forceinline__ SampleOut sample_at(const ApFrameParams& p, const ApFrameBuffers& b,
                                               double sub_i, double sub_j) {
    if constexpr (TIER == AP_TIER_FP64) {
        double x, y;
        if (p.flags & AP_FLAG_MAP_FUSED) {
            x = fma(sub_i, p.dx_hi, p.x_min_hi);
            y = fma(-sub_j, p.dy_hi, p.y_max_hi);
        } else {
            x = p.x_min_hi + sub_i * p.dx_hi;
            y = p.y_max_hi - sub_j * p.dy_hi;
        }
        return fp64_sample<ARITH>(x, y, p);
    } else if constexpr (TIER == AP_TIER_DD) {
        return dd_sample_at<ARITH>(p, sub_i, sub_j);
    } else if constexpr (TIER == AP_TIER_PERTURB) {
        return perturb_sample_at<ARITH>(p, b, sub_i, sub_j);
    } else {
        return floatexp_sample_at<ARITH>(p, b, sub_i, sub_j);
    }
}

// hist_resolve = 0: mandelbrot_unified_*_kernel semantics
//   (math_core/cuda_kernels.py:1615-1917);
// hist_resolve = 1: ssaa_resolve_hist_*_kernel semantics
//   (math_core/cuda_kernels.py:2038-2234).
template <int TIER, int ARITH>
__global__ void __launch_bounds__(kTile * kTile) render_pass_kernel(const ApFrameParams p,
                                                          const ApFrameBuffers b,
                                                          const int hist_resolve) {
    const int i = blockIdx.x * kTile + (threadIdx.x & (kTile - 1));
    const int j = blockIdx.y * kTile + (threadIdx.x / kTile);
    if (i >= p.width || j >= p.height) return;
    const size_t idx = (size_t)j * p.width + i;
    if (p.rebase_pass > 0 && b.glitch_in[idx] == 0) return;
    int mode = p.mode;
    if (hist_resolve) {
        if (p.rebase_pass == 0 && b.edge_mask[idx] == 0) return;
        mode = AP_MODE_FULL;
    } else if (mode == AP_MODE_EDGE && b.edge_mask[idx] == 0) {
        return;
    }
    constexpr bool kPert = (TIER >= AP_TIER_PERTURB);
    const bool hist_colour = hist_resolve || (p.flags & AP_FLAG_HIST_COLOUR);
    const int f = p.factor;

    if (mode == AP_MODE_COARSE) {
        const double sub_offset = ((double)f - 1.0) * 0.5;
        const SampleOut o = sample_at<TIER, ARITH>(p, b, (double)(i * f) + sub_offset,
                                                   (double)(j * f) + sub_offset);
        b.iter_map[idx] = o.s;
        if (b.kmap) b.kmap[idx] = o.k;
        if (b.s64) b.s64[idx] = o.s64;
        if (b.counters) {
            reinterpret_cast<int4*>(b.counters)[idx] = make_int4(o.iters, o.leaps, o.iters2, 0);
        }
        if (kPert && b.glitch_out) b.glitch_out[idx] = o.glitch > 0 ? 1 : 0;
        if (!(p.flags & AP_FLAG_NO_RGB)) {
            double r = 0.0, g = 0.0, bb = 0.0;
            if ((double)o.s >= 0.0) colour_of(p, b.lut, b.cdf, hist_colour, (double)o.s, r, g, bb);
            store_rgb(b.rgb, p.is_hdr, idx, r, g, bb);
        }
        return;
    }

    double ra = 0.0, ga = 0.0, ba = 0.0;
    int glitches = 0, iters = 0, leaps = 0, iters2 = 0;
    SampleOut last = interior_sample();
    for (int sy = 0; sy < f; ++sy) {
        for (int sx = 0; sx < f; ++sx) {
            const SampleOut o =
                sample_at<TIER, ARITH>(p, b, (double)(i * f + sx), (double)(j * f + sy));
            last = o;
            iters += o.iters;
            leaps += o.leaps;
            iters2 += o.iters2;
            if (o.glitch > 0) ++glitches;
            if ((double)o.s >= 0.0) {
                double r, g, bb;
                colour_of(p, b.lut, b.cdf, hist_colour, (double)o.s, r, g, bb);
                ra += r;
                ga += g;
                ba += bb;
            }
        }
    }
    const double inv = 1.0 / (double)(f * f);
    store_rgb(b.rgb, p.is_hdr, idx, ra * inv, ga * inv, ba * inv);
    if (kPert && b.glitch_out) b.glitch_out[idx] = glitches > 0 ? 1 : 0;
    if (b.counters) {
        reinterpret_cast<int4*>(b.counters)[idx] = make_int4(iters, leaps, iters2, 0);
    }
    const bool write_iter =
        hist_resolve ? (p.rebase_pass > 0) : ((p.flags & AP_FLAG_ITER_LAST_SUB) != 0);
    if (write_iter) {
        b.iter_map[idx] = last.s;
        if (b.kmap) b.kmap[idx] = last.k;
        if (b.s64) b.s64[idx] = last.s64;
    }
}

template <int TIER, int ARITH>
static int launch_pass(const ApFrameParams& p, const ApFrameBuffers& b, int hist_resolve,
                       cudaStream_t st) {
    dim3 grid((p.width + kTile - 1) / kTile, (p.height + kTile - 1) / kTile);
    render_pass_kernel<TIER, ARITH><<<grid, kTile * kTile, 0, st>>>(p, b, hist_resolve);
    return check_launch("render_pass_kernel");
}

template <int TIER>
static int launch_arith(const ApFrameParams& p, const ApFrameBuffers& b, int hist_resolve,
                        cudaStream_t st) {
    if (p.arith == AP_ARITH_REF_CPU) return launch_pass<TIER, AP_ARITH_REF_CPU>(p, b, hist_resolve, st);
    // AP_ARITH_FAST passes are one-pass rebasing passes: rebase_sample_at reads p.arith
    return launch_pass<TIER, AP_ARITH_REF_CUDA>(p, b, hist_resolve, st);
}

int validate_frame(const ApFrameParams* p, const ApFrameBuffers* b, int hist_resolve) {
    if (!p || !b) {
        set_error("null params or buffers");
        return AP_E_INVALID;
    }
    if (p->width <= 0 || p->height <= 0 || p->factor < 1 || p->max_iter < 0) {
        set_error("bad frame geometry %dx%d factor %d max_iter %d", p->width, p->height, p->factor,
                  p->max_iter);
        return AP_E_INVALID;
    }
    if ((long long)p->width * p->factor > (1LL << 24) || (long long)p->height * p->factor > (1LL << 24)) {
        set_error("sub-sample grid too large");
        return AP_E_INVALID;
    }
    if (p->fractal_type < 0 || p->fractal_type > 4) {
        set_error("fractal_type %d outside 0..4", p->fractal_type);
        return AP_E_INVALID;
    }
    if (p->fractal_type == 4 && (p->gen_n < 0 || p->gen_n > 64)) {
        set_error("gen_n %d outside 0..64", p->gen_n);
        return AP_E_INVALID;
    }
    if (p->tier < AP_TIER_FP64 || p->tier > AP_TIER_FLOATEXP32) {
        set_error("unknown tier %d", p->tier);
        return AP_E_INVALID;
    }
    if (p->arith != AP_ARITH_REF_CPU && p->arith != AP_ARITH_REF_CUDA && p->arith != AP_ARITH_FAST) {
        set_error("unknown arithmetic profile %d", p->arith);
        return AP_E_INVALID;
    }
    if (p->arith == AP_ARITH_FAST && !(p->flags & AP_FLAG_REBASE)) {
        set_error("AP_ARITH_FAST serves one-pass rebasing passes (AP_FLAG_REBASE) only");
        return AP_E_UNSUPPORTED;
    }
    if (p->mode < AP_MODE_COARSE || p->mode > AP_MODE_EDGE) {
        set_error("unknown mode %d", p->mode);
        return AP_E_INVALID;
    }
    if (!b->iter_map) {
        set_error("iter_map is required");
        return AP_E_INVALID;
    }
    if (b->counters && (reinterpret_cast<uintptr_t>(b->counters) & 15u)) {
        set_error("counters must be 16-byte aligned");
        return AP_E_INVALID;
    }
    const bool need_rgb = hist_resolve || p->mode != AP_MODE_COARSE || !(p->flags & AP_FLAG_NO_RGB);
    if (need_rgb && (!b->rgb || !b->lut)) {
        set_error("rgb and lut are required");
        return AP_E_INVALID;
    }
    const bool hist = hist_resolve || (p->flags & AP_FLAG_HIST_COLOUR);
    if (hist && (!b->cdf || p->num_bins < 2)) {
        set_error("histogram colouring needs cdf and num_bins >= 2");
        return AP_E_INVALID;
    }
    if ((p->mode == AP_MODE_EDGE || (hist_resolve && p->rebase_pass == 0)) && !b->edge_mask) {
        set_error("edge_mask is required");
        return AP_E_INVALID;
    }
    if (p->rebase_pass > 0 && !b->glitch_in) {
        set_error("glitch_in is required on rebase passes");
        return AP_E_INVALID;
    }
    if (p->flags & AP_FLAG_REBASE) {
        if (p->tier != AP_TIER_PERTURB && p->tier != AP_TIER_FLOATEXP32) {
            set_error("AP_FLAG_REBASE serves the FP64-delta and FP32 FloatExp tiers (AP_TIER_PERTURB, AP_TIER_FLOATEXP32)");
            return AP_E_UNSUPPORTED;
        }
        if (p->fractal_type == 2 || p->fractal_type == 3) {
            set_error("AP_FLAG_REBASE serves orbits that start at 0 (fractal_type 0, 1, 4)");
            return AP_E_UNSUPPORTED;
        }
        if (p->ref_len < 1 || p->rebase_pass != 0) {
            set_error("AP_FLAG_REBASE needs ref_len >= 1 and rebase_pass 0");
            return AP_E_INVALID;
        }
    }
    if (p->tier >= AP_TIER_PERTURB) {
        if (!b->ref_re || !b->ref_im || p->ref_len < 0) {
            set_error("perturbation tiers need the reference orbit");
            return AP_E_INVALID;
        }
        if (p->bla_levels > 0 && (!b->bla || p->bla_levels > 31)) {
            set_error("bla_levels %d needs a table with at most 31 levels", p->bla_levels);
            return AP_E_INVALID;
        }
    }
    return AP_OK;
}

static int dispatch(const ApFrameParams* p, const ApFrameBuffers* b, int hist_resolve,
                    void* stream) {
    int rc = validate_frame(p, b, hist_resolve);
    if (rc != AP_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (p->tier == AP_TIER_FLOATEXP32) {
        if (hist_resolve) {
            set_error("histogram resolve passes use the FP64 tiers");
            return AP_E_UNSUPPORTED;
        }
        return launch_fe32(*p, *b, st);
    }
    if (!hist_resolve) {
        rc = launch_perturb_fast(*p, *b, st);
        if (rc != AP_E_UNSUPPORTED) return rc;
    }
    switch (p->tier) {
    case AP_TIER_FP64: return launch_arith<AP_TIER_FP64>(*p, *b, hist_resolve, st);
    case AP_TIER_DD: return launch_arith<AP_TIER_DD>(*p, *b, hist_resolve, st);
    case AP_TIER_PERTURB: return launch_arith<AP_TIER_PERTURB>(*p, *b, hist_resolve, st);
    case AP_TIER_FLOATEXP: return launch_arith<AP_TIER_FLOATEXP>(*p, *b, hist_resolve, st);
    default:
        set_error("tier %d is not served by ap_render_pass", p->tier);
        return AP_E_UNSUPPORTED;
    }
}

}  // namespace ap

extern "C" int ap_render_pass(const ApFrameParams* p, const ApFrameBuffers* b, void* stream) {
    return ap::dispatch(p, b, 0, stream);
}

extern "C" int ap_resolve_hist_pass(const ApFrameParams* p, const ApFrameBuffers* b, void* stream) {
    return ap::dispatch(p, b, 1, stream);
}

extern "C" int ap_render_rows(const ApFrameParams* p, const ApFrameBuffers* b, int32_t row0, int32_t rows,
                              void* stream) {
    int rc = ap::validate_frame(p, b, 0);
    if (rc != AP_OK) return rc;
    if (row0 < 0 || rows < 0 || (long long)row0 + rows > p->height) {
        ap::set_error("ap_render_rows: rows [%d, %d) outside the frame's %d rows", row0, row0 + rows, p->height);
        return AP_E_INVALID;
    }
    rc = ap::launch_perturb_fast_rows(*p, *b, row0, rows, static_cast<cudaStream_t>(stream));
    if (rc == AP_E_UNSUPPORTED)
        ap::set_error("ap_render_rows serves coarse AP_TIER_PERTURB passes without in-kernel colour on "
                      "packed inputs (ap_pack_orbit, ap_pack_bla)");
    return rc;
}
