/*
 * apeiron_b200.h -- C ABI of the B200 escape-time engine.
 *
 * Plain structs, device pointers and sizes; every call returns 0 on success
 * or a negative AP_E_* code, with a message retrievable through
 * ap_last_error().  All launches go to the caller's cudaStream_t (passed as
 * void*; NULL means the legacy default stream) and never synchronise it.
 *
 * The entry points replace the Numba CUDA kernel launches that
 * math_core/engine.py issues from render_frame_ssaa (math_core/engine.py:1339)
 * and recolor_frame (math_core/engine.py:2138).  Each declaration cites the
 * reference kernel(s) it stands in for.
 */
#ifndef APEIRON_B200_H
#define APEIRON_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define AP_API __attribute__((visibility("default")))
#else
#define AP_API
#endif

#define AP_ABI_VERSION 7

/* Return codes. */
#define AP_OK 0
#define AP_E_INVALID (-1)   /* bad argument (null pointer, size, enum) */
#define AP_E_CUDA (-2)      /* a CUDA runtime call failed */
#define AP_E_UNSUPPORTED (-3)

/* Precision tiers, chosen by the host exactly as math_core/engine.py:1402-1408. */
#define AP_TIER_FP64 0      /* direct FP64 iteration            (cuda_kernels.py:264) */
#define AP_TIER_DD 1        /* direct double-double iteration   (cuda_kernels.py:321) */
#define AP_TIER_PERTURB 2   /* FP64-delta perturbation (+BLA)   (cuda_kernels.py:422, :594) */
#define AP_TIER_FLOATEXP 3  /* FP64-mantissa FloatExp deltas    (cuda_kernels.py:819, :1102) */
#define AP_TIER_FLOATEXP32 4 /* FP32-mantissa FloatExp deltas (this engine's fast form; all five
                                formulas, coarse passes; with or without AP_FLAG_REBASE) */

/* Arithmetic profiles.  The escape step of a boundary pixel depends on which
 * multiply-adds are fused, so the engine can reproduce either reference. */
#define AP_ARITH_REF_CPU 0   /* the reference's Numba CPU kernels as compiled (x86-64, FMA where LLVM fused) */
#define AP_ARITH_REF_CUDA 1  /* the reference's CUDA sources: explicit cuda.fma fused, nothing else */
#define AP_ARITH_FAST 2      /* the engine's own fused form of the one-pass rebasing step (AP_FLAG_REBASE
                                only; no reference counterpart): 2 Z + dz, the step and |dz|^2 each
                                as fused multiply-adds, leaps as AP_ARITH_REF_CUDA */

/* Launch modes of the unified render pass (cuda_kernels.py:1615-1917). */
#define AP_MODE_COARSE 0     /* one centred sample per pixel -> iter map + RGB */
#define AP_MODE_FULL 1       /* f x f samples for every selected pixel (rebase passes) */
#define AP_MODE_EDGE 2       /* f x f samples only where edge_mask != 0 */

/* ApFrameParams.flags */
#define AP_FLAG_NO_RGB 1u          /* skip the RGB write (histogram first pass) */
#define AP_FLAG_ESCAPE_GLITCH 2u   /* flag escapes with |Z|^2 < 4 (non-BLA sample, cuda_kernels.py:467) */
#define AP_FLAG_NAN_GUARD 4u       /* stage-2 NaN/Inf -> (k, glitch) (cuda_kernels.py:771) */
#define AP_FLAG_ITER_LAST_SUB 8u   /* supersample passes write the last sub-sample to the iter map */
#define AP_FLAG_MAP_FUSED 16u      /* pixel -> c mapping as fma(i, dx, x_min) */
#define AP_FLAG_HIST_COLOUR 32u    /* colour through the CDF table (scheme 11 resolve passes) */
/* One-pass rebasing (AP_TIER_PERTURB and AP_TIER_FLOATEXP32, fractal types 0, 1, 4; no counterpart in the
 * reference, which rebases by whole re-render passes, math_core/engine.py:1890-2113).
 * Each pixel keeps its own iteration count n and a reference index m.  When
 * |Z_m + dz| < |dz| (the delta has outgrown the value it perturbs) or the reference
 * ends (m == ref_len), the delta restarts from the orbit's start: dz <- Z_m + dz,
 * m <- 0 (Zhuoran, fractalforums.org 2021).  No pixel is flagged glitched (only a
 * NaN/Inf delta is), there is no direct-iteration stage, and rebase_pass must be 0. */
#define AP_FLAG_REBASE 64u

typedef struct ApFrameParams {
    int32_t width, height;     /* output pixels */
    int32_t factor;            /* SSAA factor f >= 1 */
    int32_t max_iter;
    int32_t fractal_type;      /* 0 Mandelbrot, 1 Burning Ship, 2 Julia, 3 BS-Julia, 4 Multibrot */
    int32_t tier;              /* AP_TIER_* */
    int32_t arith;             /* AP_ARITH_* */
    int32_t mode;              /* AP_MODE_* */
    uint32_t flags;            /* AP_FLAG_* */
    int32_t gen_n;             /* Multibrot power */
    /* Direct tiers: top-left sample and sub-sample steps (double-double; FP64 uses _hi). */
    double x_min_hi, x_min_lo, y_max_hi, y_max_lo;
    double dx_hi, dx_lo, dy_hi, dy_lo;
    /* Formula parameters. */
    double julia_cx_hi, julia_cx_lo, julia_cy_hi, julia_cy_lo;
    double gen_kr, gen_ki;
    /* Perturbation tiers: reference position (sub-sample units) and its c. */
    double ref_px, ref_py;
    double ref_cx, ref_cy;
    int32_t ref_len;           /* reference escape step; orbit arrays hold ref_len + 1 entries */
    int32_t e_scale;           /* FloatExp exponent scale (config.py:51) */
    int32_t bla_levels;        /* rows of the BLA table, 0 = no leaps */
    int32_t strict_glitch;     /* Pauldelbrot test on/off */
    int32_t rebase_pass;       /* > 0: only pixels with glitch_in != 0 are evaluated */
    int32_t bbsa_skip;         /* series-approximation skip (0 = off) */
    double bbsa_inv_r;
    double bbsa[16];           /* A..H coefficients, re/im interleaved (ar, ai, br, bi, ...) */
    /* Colouring. */
    int32_t scheme_id;         /* 0..11 (cuda_kernels.py:171) */
    int32_t num_bins;          /* CDF bins for scheme 11 (65536) */
    double palette_offset, color_density, color_contrast;
    float edge_threshold;
    int32_t is_hdr;            /* rgb is uint16 when nonzero */
} ApFrameParams;

typedef struct ApFrameBuffers {
    const double* ref_re;      /* [ref_len + 1] */
    const double* ref_im;      /* [ref_len + 1] */
    const double* bla;         /* [bla_levels, ref_len, 5]: A_re, A_im, B_re, B_im, r^2 */
    const float* lut;          /* [2048, 3] */
    const float* cdf;          /* [num_bins] normalised CDF (scheme 11) */
    const uint8_t* glitch_in;  /* [H, W] */
    const uint8_t* edge_mask;  /* [H, W] */
    float* iter_map;           /* [H, W] smooth value, float32, -1 = interior */
    void* rgb;                 /* [H, W, 3] uint8 or uint16 */
    uint8_t* glitch_out;       /* [H, W] */
    int32_t* kmap;             /* optional [H, W]: escape step; -1 never escaped, -2 cardioid/bulb skip */
    double* s64;               /* optional [H, W]: smooth value in float64, -1 = interior */
    int32_t* counters;         /* optional [H, W, 4]: work done for the pixel by this pass, summed
                                  over its sub-samples: [0] iterations stepped one at a time
                                  (direct tiers; perturbation stage 1), [1] BLA leaps taken,
                                  [2] perturbation stage-2 (direct) steps, [3] rebases
                                  (AP_FLAG_REBASE coarse passes on packed inputs; otherwise zero).  16-byte aligned;
                                  written only for pixels the pass evaluates. */
    const double* orbit_packed; /* optional [ref_len + 1, 4] from ap_pack_orbit */
    const double* bla_packed;   /* optional, from ap_pack_bla (needs orbit_packed) */
} ApFrameBuffers;

/* One tile of a batch (ap_render_batch): a coarse AP_TIER_PERTURB or AP_TIER_FLOATEXP32
 * pass on packed inputs, without in-kernel colour (p.flags has AP_FLAG_NO_RGB), with its
 * own parameters, reference orbit and outputs; single-reference, or one-pass rebasing
 * (p.flags has AP_FLAG_REBASE; fractal types 0, 1, 4).  448 bytes. */
typedef struct ApTileDesc {
    ApFrameParams p;
    const double* orbit_packed; /* ap_pack_orbit records of the tile's reference (AP_TIER_FLOATEXP32:
                                   followed by ap_pack_fe32's float records, 6 (ref_len + 1) doubles) */
    const double* bla_packed;   /* when p.bla_levels > 1: ap_pack_bla rows (AP_TIER_FLOATEXP32: ap_pack_fe32's
                                   bla_out), else NULL */
    float* iter_map;            /* [H, W] smooth values (required) */
    int32_t* kmap;              /* optional [H, W] escape steps */
    double* s64;                /* optional [H, W] float64 smooth values */
    uint8_t* glitch_out;        /* optional [H, W] glitch flags */
    int32_t* counters;          /* optional [H, W, 4] work counters, 16-byte aligned */
    int64_t reserved;
} ApTileDesc;

/* A view for the derivative entry points (FP64 direct iteration; formulas 0 Mandelbrot,
 * 2 Julia with z0 = pixel and parameter P = (pr, pi), 4 Multibrot z^n + P z + pixel).
 * Pixel (i, j) sits at (cx - w/2 + i w/(W-1), cy + h/2 - j h/(H-1)), h = w H / W.
 * 64 bytes. */
typedef struct ApGradView {
    int32_t width, height, max_iter, fractal_type, gen_n;
    int32_t ckpt_every;        /* checkpoint spacing of the orbit, 1..1024 steps */
    double cx, cy, w, pr, pi;
} ApGradView;

/* Library identity. */
AP_API int ap_abi_version(void);
AP_API const char* ap_last_error(void);

/* One unified render pass over the frame.
 * Replaces mandelbrot_unified_{fp64,dd,perturbation,floatexp}_kernel
 * (math_core/cuda_kernels.py:1615, :1666, :1736, :1827) launched from
 * math_core/engine.py:1652-1888 and the rebase relaunches at :2060, :2103. */
AP_API int ap_render_pass(const ApFrameParams* p, const ApFrameBuffers* b, void* stream);

/* Supersample/rebase resolve under histogram colouring.
 * Replaces ssaa_resolve_hist_{fp64,dd,perturbation,floatexp}_kernel
 * (math_core/cuda_kernels.py:2038-2234, launched at math_core/engine.py:1596-1635, :2048, :2092). */
AP_API int ap_resolve_hist_pass(const ApFrameParams* p, const ApFrameBuffers* b, void* stream);

/* Rows [row0, row0 + rows) of the frame p into the frame's full-size buffers (the
 * other rows are left alone): one band of a frame split across GPUs.  Each pixel is
 * evaluated exactly as ap_render_pass evaluates it (global row index, the same
 * reference position), so bands assembled from any split equal the whole frame bit
 * for bit.  Serves coarse AP_TIER_PERTURB passes without in-kernel colour on packed
 * inputs (the perturbation tiers' fast kernel); AP_E_UNSUPPORTED otherwise.  No
 * counterpart in the reference. */
AP_API int ap_render_rows(const ApFrameParams* p, const ApFrameBuffers* b, int32_t row0, int32_t rows,
                          void* stream);

/* 8-neighbour edge mask.  Replaces edge_detect_kernel (math_core/cuda_kernels.py:1587). */
AP_API int ap_edge_detect(const float* iter_map, uint8_t* edge_mask, int32_t width, int32_t height,
                   float threshold, void* stream);

/* Histogram of the iteration map followed by the normalised CDF.
 * Replaces zero_histogram_cuda_kernel, build_histogram_kernel, scan_blocks_cuda_kernel,
 * scan_single_block_cuda_kernel and finalize_normalized_cdf_cuda_kernel
 * (math_core/cuda_kernels.py:1922-2013, launched at math_core/engine.py:1435, :1576-1585).
 * hist: caller scratch of num_bins int32; cdf: num_bins float32 output. */
AP_API int ap_histogram_cdf(const float* iter_map, int32_t width, int32_t height, int32_t max_iter,
                     int32_t num_bins, int32_t* hist, float* cdf, void* stream);

/* Reference orbit in the layout the perturbation kernels read: per step the
 * 32-byte record (Z_re, Z_im, safe radius^2, level-0 BLA radius^2).  While the
 * rounded |dz|^2 is below the safe radius^2 neither the escape test, the glitch
 * test (|Z + dz|^2 < 1e-6 |Z|^2 where |Z|^2 > 1e-8, math_core/cpu_kernels.py:428-431)
 * nor the rebase test of AP_FLAG_REBASE (|Z + dz| < |dz|) can fire at that step.  The
 * last record (step ref_len) always has safe radius 0.  The level-0 radius is written by ap_pack_bla; this call
 * leaves it 0 (no leap).  out: [ref_len + 1, 4] float64. */
AP_API int ap_pack_orbit(const double* ref_re, const double* ref_im, int32_t ref_len, double* out,
                         void* stream);

/* Chained-BLA table in the layout the perturbation kernels read: the 16 radii of
 * step k in one 128-byte row ([ref_len, 16] float64), then the coefficients
 * (A_re, A_im, B_re, B_im) per step and level ([ref_len, 16, 4] float64); levels
 * at or above `levels`, and leaps that would reach the end of the orbit
 * (k + 2^d >= ref_len), hold radius 0.  table: the [levels, ref_len, 5] layout of
 * ap_build_bla.  out: 80 * ref_len float64.  orbit_packed: the ap_pack_orbit
 * records of the same orbit, whose level-0 radius slot is filled here (the coarse
 * pass tests that slot before each step; NULL leaves it 0, and no leap is taken). */
AP_API int ap_pack_bla(const double* table, int32_t levels, int32_t ref_len, double* out,
                       double* orbit_packed, void* stream);

/* Inputs of AP_TIER_FLOATEXP32 (the FP32-mantissa FloatExp fast form).
 * orbit_packed: the ap_pack_orbit records; orbit32_out: [ref_len + 1] float4 (Z_re,
 * Z_im, |Z|^2, f) in float32, f = 1 where |Z|^2 < 2^-100 (steps the kernel takes in
 * FP64) else 0, placed by convention right after the ap_pack_orbit
 * records so a frame passes one orbit_packed buffer of 6 (ref_len + 1) doubles.
 * table (optional): the ap_build_bla layout; bla_out then receives 80 ref_len
 * doubles: the radii r^2 * 2^600 as [ref_len, 16] float64 and per (step, level) a
 * 32-byte record of float mantissas (A_re, A_im, B_re, B_im) and int exponents. */
AP_API int ap_pack_fe32(const double* orbit_packed, int32_t ref_len, const double* table,
                        int32_t levels, double* orbit32_out, double* bla_out, void* stream);

/* The two halves of ap_histogram_cdf, for a frame split across GPUs: ap_histogram counts
 * (zeroing hist first) the escaped values of one band of the frame (histogram_kernel of
 * math_core/cuda_kernels.py:1999-2013); after the bands' histograms are summed (an
 * all-reduce), ap_cdf_from_histogram turns the sum into the normalised CDF exactly as
 * ap_histogram_cdf does (the float64 scan of :1929-1996).  Neither has its own
 * counterpart in the reference, which renders a frame on one GPU. */
AP_API int ap_histogram(const float* iter_map, int32_t width, int32_t height, int32_t max_iter,
                        int32_t num_bins, int32_t* hist, void* stream);
AP_API int ap_cdf_from_histogram(const int32_t* hist, int32_t num_bins, float* cdf, void* stream);

/* Largest num_bins ap_histogram_cdf_noalloc accepts (its built-in scratch, 256 KiB per GPU). */
#define AP_NOALLOC_MAX_BINS 65536

/* ap_histogram_cdf without the caller scratch: for callers that cannot allocate
 * device memory (no cudaMalloc where they run).  No counterpart in the reference.
 * The histogram goes to an array compiled into the library (AP_NOALLOC_MAX_BINS
 * int32 per GPU, held from module load until process exit); num_bins above that
 * is rejected with AP_E_INVALID.  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress), so make it before any stream capture.  The
 * address is kept for the life of the process: after cudaDeviceReset (or any other
 * teardown of the device's primary context) this entry point must not be called
 * again on that device.  All calls on a device share the array: calls that overlap
 * on the GPU race. */
AP_API int ap_histogram_cdf_noalloc(const float* iter_map, int32_t width, int32_t height,
                                    int32_t max_iter, int32_t num_bins, float* cdf, void* stream);

/* Colour every pixel from its smooth value.  With scheme 11 the CDF table is used
 * (apply_histogram_equalization_kernel, math_core/cuda_kernels.py:2016); otherwise
 * the closed-form transfer function (recolor_iter_map_cuda_kernel, :3201).  With
 * p->rebase_pass > 0 only pixels whose glitch_in is set are coloured (the pixels a
 * rebase pass re-rendered). */
AP_API int ap_colour(const ApFrameParams* p, const ApFrameBuffers* b, void* stream);

/* Write values computed elsewhere into the listed pixels: coords[n, 2] = (row, col),
 * values[n] float64 smooth values; iter_map = float32(value), RGB = the colour of the
 * float64 value (black below 0 or at or above max_iter; CDF colouring for scheme 11
 * when b->cdf is set), glitch flag cleared.  The Strict Metric re-evaluation's output
 * step (math_core/engine.py:249-266). */
AP_API int ap_set_pixels(const ApFrameParams* p, const ApFrameBuffers* b, const int32_t* coords,
                         const double* values, int32_t n, void* stream);

/* Strict Metric re-evaluation on the device (eval_glitched_pixels_cuda_kernel and
 * eval_glitched_pixels_hist_cuda_kernel, math_core/cuda_kernels.py:2450-2569; host side
 * math_core/engine.py:270-410).  Each listed pixel (coords[n, 2] = (row, col)) is
 * iterated on its own, then written like ap_set_pixels (iter_map = the float32 value,
 * RGB black for a value below 0, glitch flag cleared).
 *   AP_STRICT_DD: double-double; pixel c = x_min + col dx, y_max - row dy with the
 *     double-double view of p (x_min_hi/lo, y_max_hi/lo, dx_hi/lo, dy_hi/lo) and the
 *     Julia constant in p->julia_c{x,y}_{hi,lo}; fractal types 0-4.
 *   AP_STRICT_LIMBS: AP_STRICT_NLIMBS x 32-bit sign-magnitude fixed point (limb 0 the
 *     integer part, most significant first); signs[n, 2] (1 = negative) and
 *     limbs[n, 2, AP_STRICT_NLIMBS] give each pixel's c (x then y), v the Julia
 *     constant; fractal types 0-3 (type 4 evaluates as interior, as the reference).
 * Colours use p->arith's transfer functions and, for scheme 11, b->cdf. */
#define AP_STRICT_DD 1
#define AP_STRICT_LIMBS 2
#define AP_STRICT_FP64 3   /* views of width >= 1e-12: c = x_min_hi + col dx_hi, y_max_hi - row dy_hi
                              in FP64, iterated as compute_fp64_sample (the CUDA source form) */
#define AP_STRICT_NLIMBS 34
typedef struct ApStrictView {
    int32_t tier;
    int32_t jx_sign, jy_sign;
    int32_t reserved;
    uint32_t jx_limbs[AP_STRICT_NLIMBS];
    uint32_t jy_limbs[AP_STRICT_NLIMBS];
} ApStrictView;

AP_API int ap_strict_eval(const ApFrameParams* p, const ApFrameBuffers* b, const ApStrictView* v,
                          const int32_t* coords, const int32_t* signs, const uint32_t* limbs,
                          int32_t n, void* stream);

/* Rebase-loop statistics on the device: counts[256] (int32, zeroed here) receives the
 * number of glitched pixels in each cell of the 16 x 16 grid (row cell 16 j / H, column
 * cell 16 i / W) from which math_core/engine.py:1923-1992 picks the next reference, so
 * the host downloads 1 KB and then one cell's pixels instead of the whole maps. */
AP_API int ap_glitch_bins(const uint8_t* glitch_map, int32_t width, int32_t height, int32_t* counts,
                          void* stream);

/* Chained-BLA table from a reference orbit, built on the device.
 * Replaces _jit_build_bla_table (math_core/high_precision.py:1101) and its upload
 * (math_core/engine.py:416).  out: [levels, ref_len, 5] float64. */
AP_API int ap_build_bla(const double* ref_re, const double* ref_im, int32_t ref_len, int32_t fractal_type,
                 double tol, int32_t levels, int32_t gen_n, double gen_kr, double gen_ki,
                 double* out, void* stream);

/* The same table with the dc-aware merge of the published chained-BLA method
 * (Zhuoran, fractalforums.org 2021): a merged leap is valid while
 * |dz| < min(r1, (r2 - |B1| dc_max) / |A1|), dc_max being the largest |dc| of the
 * frame; level 0 is ap_build_bla's with tol = eps.  The reference's merge
 * (high_precision.py:1195-1230) drops the |B1| dc term, which makes its leaps
 * inaccurate where dc dominates.  No counterpart in the reference. */
AP_API int ap_build_bla_dc(const double* ref_re, const double* ref_im, int32_t ref_len,
                           int32_t fractal_type, double eps, double dc_max, int32_t levels,
                           int32_t gen_n, double gen_kr, double gen_ki, double* out, void* stream);

/* Series-approximation ("BBSA") start for the perturbation tier, computed on the HOST
 * from the host copy of the reference orbit (no device work).  Replaces
 * compute_bbsa_coeffs / _jit_compute_bbsa_coeffs (math_core/high_precision.py:50-578,
 * called from math_core/engine.py:426-470).  out[17]: out[0] = number of steps the
 * start skips, out[1..16] = (a1_re, a1_im, ..., a8_re, a8_im) for ApFrameParams.bbsa;
 * all zero where the reference returns no start (types other than 0, 2 and Multibrot
 * n = 3, order 32, e_scale > 0, bad radius). */
AP_API int ap_bbsa_coeffs(const double* ref_re, const double* ref_im, int32_t ref_len, double max_r,
                          int32_t fractal_type, double tol, int32_t order, int32_t gen_n,
                          double gen_kr, double gen_ki, int32_t e_scale, double* out);

/* Reference orbit of one point on the HOST, in binary fixed point.  Replaces the
 * Decimal orbit loop of compute_single_highprec_orbit (math_core/high_precision.py:706-875)
 * and, with escape_only, of compute_highprec_escape_scalar (:581-703).
 * seeds: 6 numbers (z0_re, z0_im, c_re, c_im, K_re, K_im), each `limbs` little-endian
 * uint64 limbs of two's-complement fixed point value * 2^(64 (limbs - int_limbs));
 * limbs <= 160; int_limbs >= ceil((16 n + 9) / 64) (n = 2 except Multibrot), so that
 * |Z|^2 of the first escaped Z is representable.
 * escape_only = 0: ref_re/ref_im (max_iter + 1 float64 each) receive the orbit rounded
 * to nearest, *ref_len the step at which |Z|^2 > 65536 (max_iter if none; an exactly
 * repeating Mandelbrot/Julia orbit found at power-of-two checkpoints is copied to the
 * end).  escape_only = 1: no arrays, *ref_len = escape step.  escape_mag2 (optional):
 * |Z|^2 at the escape step, rounded to float64 (left as is when the orbit never escapes).
 * trace_hash (optional): a hash of the float64 values of every Z_k up to the escape, so
 * that runs at two precisions can confirm they followed the same float64 trajectory. */
AP_API int ap_reference_orbit(const uint64_t* seeds, int32_t limbs, int32_t int_limbs,
                              int32_t fractal_type,
                              int32_t gen_n, int32_t max_iter, int32_t escape_only,
                              double* ref_re, double* ref_im, int32_t* ref_len,
                              double* escape_mag2, uint64_t* trace_hash);

/* ap_reference_orbit (escape_only = 0) with a proof against the Decimal iteration of
 * dec_digits significant digits (math_core/high_precision.py:802-873): *certified = 1 when
 * a running error bound (the Decimal roundings, 5 10^-dec_digits per operation, and this
 * run's truncations, grown by the map) shows that every stored float64 value, every
 * bailout decision and the escape |Z|^2 equal the Decimal iteration's; 0 otherwise (a
 * copied cycle, or a bound too wide somewhere), when the caller compares two precisions
 * instead.  Every fractal type; dec_digits >= 1. */
AP_API int ap_reference_orbit_cert(const uint64_t* seeds, int32_t limbs, int32_t int_limbs,
                                   int32_t fractal_type, int32_t gen_n, int32_t max_iter,
                                   int32_t dec_digits, double* ref_re, double* ref_im, int32_t* ref_len,
                                   double* escape_mag2, int32_t* certified);

/* The escape iteration of compute_highprec_escape_scalar in Decimal arithmetic
 * (math_core/high_precision.py:581-703, its decimal-module branch), on the host: for
 * the points whose fixed-point runs disagree.  Values are (-1)^neg coef 10^exp with
 * coef in base-1e8 limbs, little-endian, one per uint64.  meta: 6 x (neg, exp, n) for
 * z0_re, z0_im, c_re, c_im, K_re, K_im (any number of digits up to 1600); limbs: 6 x
 * limb_stride (<= 200).  Every +, - and * is exact, then rounded to prec significant
 * digits, half to even; abs() rounds too.  *k_out = the escape step (|Z|^2 > 65536)
 * or max_iter; mag2_meta/mag2_limbs (3 and 400 entries) = |Z|^2 there. */
AP_API int ap_decimal_escape(const int64_t* meta, const uint64_t* limbs, int32_t limb_stride,
                             int32_t prec, int32_t fractal_type, int32_t gen_n, int32_t max_iter,
                             int32_t* k_out, int64_t* mag2_meta, uint64_t* mag2_limbs);

/* The orbit loop of the same Decimal iteration (decimal_orbit, the reference orbit of
 * math_core/high_precision.py:706-875 when the fixed-point runs disagree), on the host:
 * seeds as for ap_decimal_escape; ref_re/ref_im (max_iter + 1 float64) receive float(Z_k),
 * correctly rounded; *ref_len = the escape step or max_iter; an exactly repeating
 * Mandelbrot/Julia orbit found at power-of-two checkpoints has its cycle copied to the end.
 * AP_E_UNSUPPORTED when a value's conversion is not decided by the bounds this code keeps
 * (a tie or a near-tie, a value above 2^127 or outside the normal double range): the
 * caller then iterates in the decimal module. */
AP_API int ap_decimal_orbit(const int64_t* meta, const uint64_t* limbs, int32_t limb_stride,
                            int32_t prec, int32_t fractal_type, int32_t gen_n, int32_t max_iter,
                            double* ref_re, double* ref_im, int32_t* ref_len);

/* float(Decimal) of one value (meta: neg, exp, n; limbs: n base-1e8 limbs), or
 * AP_E_UNSUPPORTED as above; for checking the conversion against the decimal module. */
AP_API int ap_decimal_to_double(const int64_t* meta, const uint64_t* limbs, double* out);

/* One operation of that arithmetic (op 0 add, 1 subtract, 2 multiply, 3 compare into
 * *cmp_out), for checking it against the decimal module; out: 3 + 400 entries. */
AP_API int ap_decimal_arith(int32_t op, const int64_t* a_meta, const uint64_t* a_limbs,
                            const int64_t* b_meta, const uint64_t* b_limbs, int32_t prec,
                            int64_t* out_meta, uint64_t* out_limbs, int32_t* cmp_out);

/* Batches (no single counterpart: the reference renders tile by tile, e.g.
 * workers/image_workers.py:428-601 calling render_frame_ssaa per tile).
 * ap_batch_plan (HOST): checks every tile of host_tiles[n] and writes first_patch[n + 1],
 * the number of each tile's first 256-pixel patch (patch_w x patch_h == 256) and the total;
 * tiles should come in decreasing order of expected cost.
 * ap_render_batch: renders all tiles with one persistent kernel of blocks_per_sm blocks per
 * SM that take pixels from a shared counter (device word *queue_head, reset here).  A block
 * works in rounds: each thread runs one pixel for `quantum` loop steps; the unfinished
 * pixels are compacted into the block's first slots (shared memory) and the slots left
 * over take the next consecutive pixels of the queue with one atomicAdd.
 * tiles and first_patch are device copies of the planned arrays.  min_blocks (4 or 6) picks
 * the register budget the kernel is compiled for; arith is the tiles' common profile
 * (AP_ARITH_FAST when the plan holds AP_ARITH_FAST tiles: one-pass tiles only, the others
 * then carry AP_ARITH_REF_CUDA; AP_TIER_FLOATEXP32 tiles compute in the FP32 form whatever
 * the profile).  Values equal ap_render_pass's for each tile. */
AP_API int ap_batch_plan(const ApTileDesc* host_tiles, int32_t n, int32_t patch_w, int32_t patch_h,
                         int64_t* first_patch);
AP_API int ap_render_batch(const ApTileDesc* tiles, const int64_t* first_patch, int32_t n,
                           int32_t arith, int32_t patch_w, int32_t patch_h, int32_t blocks_per_sm,
                           int32_t min_blocks, int32_t quantum, unsigned long long* queue_head,
                           void* stream);

/* Derivatives of the smooth escape value (no counterpart in the reference).
 * theta = (cx, cy, ln w, Re P, Im P).
 * ap_smooth_forward: s64[H, W] float64 smooth values (-1 interior), kmap[H, W] escape
 *   steps (-1 bounded, -2 cardioid/bulb), and, when ckpt is given, the orbit at every
 *   ckpt_every-th step: ckpt[H, W, n_ck] complex float64, n_ck >= ceil(max_iter/ckpt_every)+1.
 * ap_smooth_adjoint: for grad_s[H, W] = dL/ds, dL/dtheta summed per tile of 8 x 4 pixels
 *   into block_sums[ap_smooth_adjoint_blocks(W, H), 5] (the caller sums the rows); the orbit
 *   is recomputed segment by segment from ckpt, never stored; pix_grads[H, W, 5]
 *   (optional) receives each pixel's term.
 * ap_smooth_tangent: forward mode, ds[H, W, 5] = ds/dtheta per pixel. */
AP_API int ap_smooth_forward(const ApGradView* v, double* s64, int32_t* kmap, double* ckpt,
                             int32_t n_ck, void* stream);
AP_API int32_t ap_smooth_adjoint_blocks(int32_t width, int32_t height);
AP_API int ap_smooth_adjoint(const ApGradView* v, const double* grad_s, const int32_t* kmap,
                             const double* ckpt, int32_t n_ck, double* pix_grads, double* block_sums,
                             void* stream);
AP_API int ap_smooth_tangent(const ApGradView* v, double* ds, void* stream);

/* Measurement helper (no counterpart in the reference): number of kernels this
 * library has launched in the process so far. */
AP_API uint64_t ap_launch_counter(void);

/* Measurement helper (no counterpart in the reference): dependent-FMA throughput
 * probe, precision 64 or 32, blocks x 256 threads x 8 chains x iters FMAs.
 * scratch: >= blocks elements of the precision's type; *flops = FLOPs launched. */
AP_API int ap_fma_peak_launch(int32_t precision, int32_t blocks, int32_t iters, void* scratch,
                              double* flops, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* APEIRON_B200_H */
