/*
 * ap_oracle.c -- CPU restatement of the reference escape-time path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle for the CUDA engine:
 * the parity tests, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py call it; the product path never does.  It is written from the
 * reference's Python/Numba sources line by line, in plain C, and shares no
 * code with the CUDA kernels.
 *
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off -pthread).  Implicit
 * contraction is disabled, so every fused multiply-add below is written out
 * with fma() exactly where the reference computes one:
 *
 *   AP_ARITH_REF_CPU   the reference's Numba CPU kernels as compiled here by
 *                      LLVM for x86-64 (fastmath functions contract some
 *                      multiply-adds and reassociate a few sums; the fused
 *                      forms below were read off that compiled code).
 *   AP_ARITH_REF_CUDA  the reference's CUDA sources as written: cuda.fma is
 *                      fused, every other operation is rounded separately.
 *
 * Two forms have no reference counterpart and are restated from the engine's
 * own definitions, so that device frames can be pinned bit for bit: the fused
 * one-pass rebasing step (AP_ARITH_FAST) and the FP32-mantissa FloatExp form
 * (AP_TIER_FLOATEXP32).  Where their precision carries a view, their values
 * equal the reference's goldens (tests/test_oracle_rebase.py,
 * tests/test_oracle_fe32.py).
 *
 * Parity is pinned by the .npz fixtures in tests/golden, generated by running the reference
 * (tests/golden/make_golden.py).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "apeiron_b200.h"

#define APO_EXPORT __attribute__((visibility("default")))

/* ---- row-parallel helper (pthreads; rows are handed out one at a time) ---- */
typedef void (*row_fn)(void* ctx, int row);
typedef struct {
    row_fn fn;
    void* ctx;
    int rows;
    int next;
    pthread_mutex_t lock;
} RowPool;

static void* row_worker(void* arg) {
    RowPool* rp = (RowPool*)arg;
    for (;;) {
        pthread_mutex_lock(&rp->lock);
        int r = rp->next++;
        pthread_mutex_unlock(&rp->lock);
        if (r >= rp->rows) break;
        rp->fn(rp->ctx, r);
    }
    return NULL;
}

static int g_threads = 0; /* 0: all online cores */

static void parallel_rows(int rows, row_fn fn, void* ctx) {
    int n = g_threads > 0 ? g_threads : (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (n < 1) n = 1;
    if (n > 256) n = 256;
    if (n > rows) n = rows;
    RowPool rp = {fn, ctx, rows, 0, PTHREAD_MUTEX_INITIALIZER};
    if (n <= 1) {
        row_worker(&rp);
        return;
    }
    pthread_t th[256];
    int started = 0;
    for (int t = 1; t < n; t++)
        if (pthread_create(&th[started], NULL, row_worker, &rp) == 0) started++;
    row_worker(&rp);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
}

/* config.py:25-26 (passed by the engine to every kernel as doubles). */
static const double INV_LN2 = 1.4426950408889634;
static const double LN_BAILOUT_LOG = 1.7129177284488854;
static const double BAILOUT = 65536.0;

typedef struct {
    float s;      /* float32 smooth value as the reference stores it; -1 interior */
    double s64;   /* the same quantity in float64 */
    int k;        /* escape step, -1 never escaped */
    int glitch;
} Sample;

/* Python's float modulo for a positive divisor (x % m). */
static double py_mod(double x, double m) {
    double r = fmod(x, m);
    if (r != 0.0) {
        if ((r < 0.0) != (m < 0.0)) r += m;
    } else {
        r = copysign(0.0, m);
    }
    return r;
}

/* 1/ln(n) rounded to float32 for Multibrot, else 1/ln 2 (cpu_kernels.py:241). */
static double inv_ln_for(int fractal_type, int gen_n) {
    if (fractal_type == 4 && gen_n > 1) return (double)(float)(1.0 / log((double)gen_n));
    return INV_LN2;
}

/* Smooth escape value: f32(k+1) - f32(nu) (cpu_kernels.py:249, cuda_kernels.py:280). */
static Sample escaped(int k, double mag2, double inv_ln) {
    Sample o;
    double log_mag = log(mag2);
    o.k = k;
    o.glitch = 0;
    if (log_mag > 1.0) {
        double nu = (log(0.5 * log_mag) - LN_BAILOUT_LOG) * inv_ln;
        o.s = (float)((double)k + 1.0) - (float)nu;
        o.s64 = ((double)k + 1.0) - nu;
    } else {
        o.s = (float)k;
        o.s64 = (double)k;
    }
    return o;
}

static Sample interior(void) {
    Sample o;
    o.s = -1.0f;
    o.s64 = -1.0;
    o.k = -1;
    o.glitch = 0;
    return o;
}

/* Removed by the Mandelbrot cardioid/bulb test: interior with zero iterations. */
static Sample skipped(void) {
    Sample o = interior();
    o.k = -2;
    return o;
}

/* ------------------------------------------------------------------------- */
/* FP64 direct iteration: cpu_kernels.py:228-266 / cuda_kernels.py:264-317    */
/* ------------------------------------------------------------------------- */
static Sample fp64_sample(double x, double y, const ApFrameParams* p) {
    const int ft = p->fractal_type;
    const int cpu = (p->arith == AP_ARITH_REF_CPU);
    const int max_iter = p->max_iter;
    double zx, zy, cx, cy;

    if (ft == 0) {
        /* Main cardioid and period-2 bulb. */
        double xm = x - 0.25;
        double y2 = y * y;
        double q = cpu ? fma(xm, xm, y2) : xm * xm + y2;
        double xp = x + 1.0;
        double b = cpu ? fma(xp, xp, y2) : xp * xp + y2;
        if ((q * (q + xm) <= 0.25 * y2) || (b <= 0.0625)) return skipped();
    }
    if (ft == 2 || ft == 3) {
        zx = x; zy = y; cx = p->julia_cx_hi; cy = p->julia_cy_hi;
    } else {
        zx = 0.0; zy = 0.0; cx = x; cy = y;
    }
    const double inv_ln = inv_ln_for(ft, p->gen_n);

    if (ft == 0 || ft == 2) {
        for (int k = 0; k < max_iter; k++) {
            double zx2 = zx * zx, zy2 = zy * zy;
            double mag2 = zx2 + zy2;
            if (mag2 > BAILOUT) return escaped(k, mag2, inv_ln);
            if (cpu) {
                /* zy' = fma(2zy, zx, cy); zx' = (cx - zy^2) + zx^2 */
                double nzy = fma(zy + zy, zx, cy);
                zx = (cx - zy2) + zx2;
                zy = nzy;
            } else {
                zy = 2.0 * zx * zy + cy;
                zx = zx2 - zy2 + cx;
            }
        }
        return interior();
    } else if (ft == 1 || ft == 3) {
        for (int k = 0; k < max_iter; k++) {
            double zx2 = zx * zx, zy2 = zy * zy;
            double mag2 = zx2 + zy2;
            if (mag2 > BAILOUT) return escaped(k, mag2, inv_ln);
            double ax = fabs(zx), ay = fabs(zy);
            if (cpu) {
                /* zy' = fma(|zx|, 2|zy|, -cy); zx' = (cx + zx^2) - zy^2 */
                double nzy = fma(ax, ay + ay, -cy);
                zx = (cx + zx2) - zy2;
                zy = nzy;
            } else {
                zy = 2.0 * ax * ay - cy;
                zx = zx2 - zy2 + cx;
            }
        }
        return interior();
    } else if (ft == 4) {
        const int n = p->gen_n;
        const double kr = p->gen_kr, ki = p->gen_ki;
        for (int k = 0; k < max_iter; k++) {
            double mag2;
            if (cpu) {
                mag2 = fma(zx, zx, zy * zy);
            } else {
                double zx2 = zx * zx, zy2 = zy * zy;
                mag2 = zx2 + zy2;
            }
            if (mag2 > BAILOUT) return escaped(k, mag2, inv_ln);
            double zr = zx, zi = zy;
            for (int t = 0; t < n - 1; t++) {
                double nr, ni;
                if (cpu) {
                    nr = fma(zr, zx, -(zi * zy));
                    ni = fma(zi, zx, zr * zy);
                } else {
                    nr = zr * zx - zi * zy;
                    ni = zr * zy + zi * zx;
                }
                zr = nr; zi = ni;
            }
            if (cpu) {
                /* zx' = fma(zx, kr, -fma(ki, zy, -cx)) + zn_r ; zy' = fma(ki, zx, fma(zy, kr, cy)) + zn_i */
                double a = fma(zx, kr, -fma(ki, zy, -cx));
                double b = fma(ki, zx, fma(zy, kr, cy));
                zx = a + zr;
                zy = b + zi;
            } else {
                double kz_r = kr * zx - ki * zy;
                double kz_i = kr * zy + ki * zx;
                zx = zr + kz_r + cx;
                zy = zi + kz_i + cy;
            }
        }
        return interior();
    }
    return interior();
}

/* ------------------------------------------------------------------------- */
/* Colouring: cuda_kernels.py:157-259                                         */
/* ------------------------------------------------------------------------- */
static double tri_wave(double phase) {
    return 1.0 - fabs((phase < 0.0 ? phase + 2.0 : phase) - 1.0);
}

/* sqrt of the smooth value: the CPU reference holds it as float32 and Numba
 * evaluates math.sqrt(float32) in float32; the CUDA reference holds float64. */
static double sqrt_s(double s, int f32) { return f32 ? (double)sqrtf((float)s) : sqrt(s); }

static double palette_norm(double s, int scheme, double off, double density, double contrast, int f32) {
    const double dens = density <= 0.0 ? 1.0 : density;
    const double cont = contrast <= 0.0 ? 1.0 : contrast;
    const double TWO_PI = 6.28318530718;
    if (scheme == 0 || scheme > 10) {
        double tri = tri_wave(py_mod(sqrt_s(s, f32) * (0.125 * dens) + off * 2.0, 2.0));
        return cont != 1.0 ? pow(tri, cont) : tri;
    } else if (scheme == 1) {
        return tri_wave(py_mod(log(s * cont + 1.0) * (0.45 * dens) + off * 2.0, 2.0));
    } else if (scheme == 2) {
        double tri = tri_wave(py_mod(sqrt_s(s, f32) * (0.125 * dens) + off * 2.0, 2.0));
        double k = 4.0 * cont;
        double td = tanh(0.5 * k);
        double scale = fabs(td) > 1e-7 ? 0.5 / td : 0.5186574;
        return 0.5 + tanh((tri - 0.5) * k) * scale;
    } else if (scheme == 3) {
        double tri = tri_wave(py_mod(sqrt_s(s, f32) * (0.125 * dens) + off * 2.0, 2.0));
        double k = 3.0 * cont;
        double ed = exp(k) - 1.0;
        double scale = fabs(ed) > 1e-7 ? 1.0 / ed : 0.0523957;
        return (exp(k * tri) - 1.0) * scale;
    } else if (scheme == 4) {
        double tri = tri_wave(py_mod(sqrt_s(s, f32) * (0.5 * dens) + off * 2.0, 2.0));
        return cont != 1.0 ? pow(tri, cont) : tri;
    } else if (scheme == 5) {
        double ang = s * (0.05 * dens) + off * TWO_PI;
        double ratio = 1.61803398875 * cont;
        return 0.5 + 0.25 * (sin(ang) + sin(ang * ratio));
    } else if (scheme == 6) {
        double ang = s * (0.08 * dens) + off * TWO_PI;
        double val = 0.5 * (1.0 - cos(ang));
        return cont != 1.0 ? pow(val, cont) : val;
    } else if (scheme == 7) {
        double ph = s * (0.05 * dens) + off * TWO_PI;
        double b = 0.5 * cont;
        double wave = sin(ph) + b * sin(ph * 2.0 + 1.2) + (b * b) * sin(ph * 4.0 + 2.4) +
                      (b * b * b) * sin(ph * 8.0 + 3.6);
        double ns = 1.0 + b + b * b + b * b * b;
        double scale = ns > 1e-7 ? 0.5 / ns : 0.26666666666666666;
        return 0.5 + scale * wave;
    } else if (scheme == 8) {
        double tri = tri_wave(py_mod(sqrt_s(s, f32) * (0.1 * dens) + off * 2.0, 2.0));
        if (cont != 1.0) tri = pow(tri, cont);
        double t2 = tri * tri;
        return t2 * tri * (tri * (tri * 6.0 - 15.0) + 10.0);
    } else if (scheme == 9) {
        double ang = s * (0.04 * dens) + (s * s) * (0.00008 * dens * cont) + off * TWO_PI;
        return 0.5 + 0.5 * sin(ang);
    } else if (scheme == 10) {
        double raw = py_mod(1.0 - exp(-0.06 * cont * sqrt(s * dens)) + off, 1.0);
        return raw >= 0.0 ? raw : raw + 1.0;
    }
    return 0.0;
}

/* cuda_kernels.py:237-259 */
static double cdf_norm(double s, int max_iter, const float* cdf, int num_bins,
                       double off, double density, double contrast) {
    if (s < 0.0) return -1.0;
    double inv_max = 1.0 / fmax(1.0, (double)max_iter);
    double pos = (s * inv_max) * (double)(num_bins - 1);
    int k = (int)pos;
    double c;
    if (k >= num_bins - 1) {
        c = cdf[num_bins - 1];
    } else if (k < 0) {
        c = cdf[0];
    } else {
        double frac = pos - (double)k;
        float c0 = cdf[k], c1 = cdf[k + 1];
        float d = c1 - c0;                 /* float32 difference */
        c = (double)c0 + frac * (double)d;
    }
    if (contrast != 1.0 && contrast > 0.0) c = pow(c, contrast);
    double dens = density <= 0.0 ? 1.0 : density;
    return tri_wave(py_mod(c * (2.0 * dens) + off * 2.0, 2.0));
}

/* cuda_kernels.py:157-168 */
static void lut_lerp(const float* lut, double norm, double* r, double* g, double* b) {
    double n = norm < 0.0 ? 0.0 : (norm > 1.0 ? 1.0 : norm);
    double pos = n * 2047.0;
    int i0 = (int)pos;
    int i1 = i0 >= 2047 ? 2047 : i0 + 1;
    double frac = pos - (double)i0;
    double inv = 1.0 - frac;
    *r = (double)lut[i0 * 3 + 0] * inv + (double)lut[i1 * 3 + 0] * frac;
    *g = (double)lut[i0 * 3 + 1] * inv + (double)lut[i1 * 3 + 1] * frac;
    *b = (double)lut[i0 * 3 + 2] * inv + (double)lut[i1 * 3 + 2] * frac;
}

static double colour_norm(const ApFrameParams* p, const ApFrameBuffers* bf, double s, int hist) {
    if (hist)
        return cdf_norm(s, p->max_iter, bf->cdf, p->num_bins, p->palette_offset, p->color_density,
                        p->color_contrast);
    return palette_norm(s, p->scheme_id, p->palette_offset, p->color_density, p->color_contrast,
                        p->arith == AP_ARITH_REF_CPU);
}

static void put_rgb(const ApFrameParams* p, void* rgb, size_t idx, double r, double g, double b) {
    if (p->is_hdr) {
        uint16_t* o = (uint16_t*)rgb + idx * 3;
        o[0] = (uint16_t)(int64_t)(r + 0.5);
        o[1] = (uint16_t)(int64_t)(g + 0.5);
        o[2] = (uint16_t)(int64_t)(b + 0.5);
    } else {
        uint8_t* o = (uint8_t*)rgb + idx * 3;
        o[0] = (uint8_t)(int64_t)(r + 0.5);
        o[1] = (uint8_t)(int64_t)(g + 0.5);
        o[2] = (uint8_t)(int64_t)(b + 0.5);
    }
}

/* ------------------------------------------------------------------------- */
/* Sample dispatch over the tiers                                             */
/* ------------------------------------------------------------------------- */
/* Defined further down (perturbation tiers). */
static Sample dd_sample_at(const ApFrameParams* p, double sub_i, double sub_j);
static Sample pert_sample_at(const ApFrameParams* p, const ApFrameBuffers* b, double sub_i,
                             double sub_j);
static Sample floatexp_sample_at(const ApFrameParams* p, const ApFrameBuffers* b, double sub_i,
                                 double sub_j);
static Sample fe32_sample_at(const ApFrameParams* p, const ApFrameBuffers* b, double sub_i, double sub_j);

/* Sub-sample coordinates (sub_i, sub_j) -> sample, as each unified kernel maps them. */
static Sample sample_at(const ApFrameParams* p, const ApFrameBuffers* b, double sub_i, double sub_j) {
    switch (p->tier) {
    case AP_TIER_FP64: {
        double x, y;
        if (p->flags & AP_FLAG_MAP_FUSED) {
            x = fma(sub_i, p->dx_hi, p->x_min_hi);
            y = fma(-sub_j, p->dy_hi, p->y_max_hi);
        } else {
            x = p->x_min_hi + sub_i * p->dx_hi;
            y = p->y_max_hi - sub_j * p->dy_hi;
        }
        return fp64_sample(x, y, p);
    }
    case AP_TIER_DD:
        return dd_sample_at(p, sub_i, sub_j);
    case AP_TIER_FLOATEXP:
        return floatexp_sample_at(p, b, sub_i, sub_j);
    case AP_TIER_FLOATEXP32:
        return fe32_sample_at(p, b, sub_i, sub_j);
    default:
        return pert_sample_at(p, b, sub_i, sub_j);
    }
}

static int is_perturbative(const ApFrameParams* p) {
    return p->tier == AP_TIER_PERTURB || p->tier == AP_TIER_FLOATEXP || p->tier == AP_TIER_FLOATEXP32;
}

/* One unified pass (cuda_kernels.py:1615-1917).  hist_resolve selects the
 * ssaa_resolve_hist_* semantics (cuda_kernels.py:2038-2234). */
typedef struct {
    const ApFrameParams* p;
    const ApFrameBuffers* b;
    int hist_resolve;
} PassCtx;

static void render_row(void* vctx, int j) {
    const PassCtx* c = (const PassCtx*)vctx;
    const ApFrameParams* p = c->p;
    const ApFrameBuffers* b = c->b;
    const int hist_resolve = c->hist_resolve;
    const int W = p->width, f = p->factor;
    const double sub_offset = ((double)f - 1.0) * 0.5;
    const int pert = is_perturbative(p);
    const int hist_colour = hist_resolve || (p->flags & AP_FLAG_HIST_COLOUR);
    {
        for (int i = 0; i < W; i++) {
            const size_t idx = (size_t)j * W + i;
            if (p->rebase_pass > 0 && b->glitch_in[idx] == 0) continue;
            int mode = p->mode;
            if (hist_resolve) {
                /* Resolve pass: edge pixels on pass 0, glitched pixels on rebase passes. */
                if (p->rebase_pass == 0 && b->edge_mask[idx] == 0) continue;
                mode = AP_MODE_FULL;
            } else if (mode == AP_MODE_EDGE && b->edge_mask[idx] == 0) {
                continue;
            }
            if (mode == AP_MODE_COARSE) {
                Sample o = sample_at(p, b, (double)(i * f) + sub_offset, (double)(j * f) + sub_offset);
                b->iter_map[idx] = o.s;
                if (b->kmap) b->kmap[idx] = o.k;
                if (b->s64) b->s64[idx] = o.s64;
                if (pert && b->glitch_out) b->glitch_out[idx] = o.glitch > 0 ? 1 : 0;
                if (!(p->flags & AP_FLAG_NO_RGB)) {
                    double r = 0, g = 0, bb = 0;
                    if ((double)o.s >= 0.0) {
                        lut_lerp(b->lut, colour_norm(p, b, (double)o.s, hist_colour), &r, &g, &bb);
                    }
                    put_rgb(p, b->rgb, idx, r, g, bb);
                }
            } else {
                double ra = 0.0, ga = 0.0, ba = 0.0;
                int glitches = 0;
                Sample last = interior();
                for (int sy = 0; sy < f; sy++) {
                    for (int sx = 0; sx < f; sx++) {
                        Sample o = sample_at(p, b, (double)(i * f + sx), (double)(j * f + sy));
                        last = o;
                        if (o.glitch > 0) glitches++;
                        if ((double)o.s >= 0.0) {
                            double r, g, bb;
                            lut_lerp(b->lut, colour_norm(p, b, (double)o.s, hist_colour), &r, &g, &bb);
                            ra += r; ga += g; ba += bb;
                        }
                    }
                }
                const double inv = 1.0 / (double)(f * f);
                put_rgb(p, b->rgb, idx, ra * inv, ga * inv, ba * inv);
                if (pert && b->glitch_out) b->glitch_out[idx] = glitches > 0 ? 1 : 0;
                const int write_iter = hist_resolve ? (p->rebase_pass > 0)
                                                    : ((p->flags & AP_FLAG_ITER_LAST_SUB) != 0);
                if (write_iter) {
                    b->iter_map[idx] = last.s;
                    if (b->kmap) b->kmap[idx] = last.k;
                    if (b->s64) b->s64[idx] = last.s64;
                }
            }
        }
    }
}

static void render_pass(const ApFrameParams* p, const ApFrameBuffers* b, int hist_resolve) {
    PassCtx c = {p, b, hist_resolve};
    parallel_rows(p->height, render_row, &c);
}

/* ------------------------------------------------------------------------- */
/* DD and perturbation tiers (filled in by the following sections)            */
/* ------------------------------------------------------------------------- */
/* Double-double arithmetic: cpu_kernels.py:96-153 (CPU: Dekker split) and
 * cuda_kernels.py:45-90 (CUDA: error-free product by fma). */
typedef struct { double hi, lo; } DD;

static DD dd_two_sum(double a, double b) {
    double s = a + b, v = s - a;
    DD r = {s, (a - (s - v)) + (b - v)};
    return r;
}

static DD dd_two_prod(double a, double b, int cpu) {
    DD r;
    if (cpu) {
        double c = 134217729.0 * a;
        double ah = c - (c - a), al = a - ah;
        c = 134217729.0 * b;
        double bh = c - (c - b), bl = b - bh;
        r.hi = a * b;
        r.lo = ((ah * bh - r.hi) + ah * bl + al * bh) + al * bl;
    } else {
        r.hi = a * b;
        r.lo = fma(a, b, -r.hi);
    }
    return r;
}

static DD dd_add(DD a, DD b) {
    DD s = dd_two_sum(a.hi, b.hi);
    return dd_two_sum(s.hi, s.lo + a.lo + b.lo);
}

static DD dd_sub(DD a, DD b) {
    DD s = dd_two_sum(a.hi, -b.hi);
    return dd_two_sum(s.hi, s.lo + a.lo - b.lo);
}

static DD dd_mul(DD a, DD b, int cpu) {
    DD pr = dd_two_prod(a.hi, b.hi, cpu);
    return dd_two_sum(pr.hi, pr.lo + a.hi * b.lo + a.lo * b.hi);
}

static DD dd_mul_f64(DD a, double b, int cpu) {
    DD pr = dd_two_prod(a.hi, b, cpu);
    return dd_two_sum(pr.hi, pr.lo + a.lo * b);
}

static DD dd_sqr(DD a, int cpu) {
    DD pr = dd_two_prod(a.hi, a.hi, cpu);
    return dd_two_sum(pr.hi, pr.lo + 2.0 * a.hi * a.lo);
}

static DD dd_abs(DD a) {
    if (a.hi < 0.0 || (a.hi == 0.0 && a.lo < 0.0)) {
        DD r = {-a.hi, -a.lo};
        return r;
    }
    return a;
}

/* cpu_kernels.py:271-369 / cuda_kernels.py:321-418 */
static Sample dd_sample(DD cx0, DD cy0, const ApFrameParams* p) {
    const int ft = p->fractal_type, cpu = p->arith == AP_ARITH_REF_CPU;
    if (ft == 0) {
        double xm = cx0.hi - 0.25, y2 = cy0.hi * cy0.hi;
        double q = xm * xm + y2;
        if ((q * (q + xm) <= 0.25 * y2) || ((cx0.hi + 1.0) * (cx0.hi + 1.0) + y2 <= 0.0625))
            return skipped();
    }
    DD jx = {p->julia_cx_hi, p->julia_cx_lo}, jy = {p->julia_cy_hi, p->julia_cy_lo};
    DD zero = {0.0, 0.0};
    DD zx, zy, cx, cy;
    if (ft == 2 || ft == 3) { zx = cx0; zy = cy0; cx = jx; cy = jy; }
    else { zx = zero; zy = zero; cx = cx0; cy = cy0; }
    const double inv_ln = inv_ln_for(ft, p->gen_n);
    for (int k = 0; k < p->max_iter; k++) {
        DD zx2 = dd_sqr(zx, cpu), zy2 = dd_sqr(zy, cpu);
        double mag2 = zx2.hi + zy2.hi;
        if (mag2 > BAILOUT) return escaped(k, mag2, inv_ln);
        if (ft == 0 || ft == 2) {
            DD sub = dd_sub(zx2, zy2);
            DD zxy = dd_mul(zx, zy, cpu);
            DD two = {zxy.hi * 2.0, zxy.lo * 2.0};
            zx = dd_add(sub, cx);
            zy = dd_add(two, cy);
        } else if (ft == 1 || ft == 3) {
            DD sub = dd_sub(zx2, zy2);
            DD zxy = dd_mul(dd_abs(zx), dd_abs(zy), cpu);
            DD two = {zxy.hi * 2.0, zxy.lo * 2.0};
            zx = dd_add(sub, cx);
            zy = dd_sub(two, cy);
        } else if (ft == 4) {
            DD cr = zx, ci = zy;
            for (int t = 0; t < p->gen_n - 1; t++) {
                DD r1 = dd_mul(cr, zx, cpu), r2 = dd_mul(ci, zy, cpu);
                DD re = dd_sub(r1, r2);
                DD i1 = dd_mul(cr, zy, cpu), i2 = dd_mul(ci, zx, cpu);
                DD im = dd_add(i1, i2);
                cr = re; ci = im;
            }
            DD kz_r = dd_sub(dd_mul_f64(zx, p->gen_kr, cpu), dd_mul_f64(zy, p->gen_ki, cpu));
            DD kz_i = dd_add(dd_mul_f64(zy, p->gen_kr, cpu), dd_mul_f64(zx, p->gen_ki, cpu));
            DD tr = dd_add(cr, kz_r), ti = dd_add(ci, kz_i);
            zx = dd_add(tr, cx);
            zy = dd_add(ti, cy);
        } else {
            return interior();
        }
    }
    return interior();
}

/* Pixel mapping of the DD kernels (cuda_kernels.py:1685-1691). */
static Sample dd_sample_at(const ApFrameParams* p, double sub_i, double sub_j) {
    const int cpu = p->arith == AP_ARITH_REF_CPU;
    DD dy = {p->dy_hi, p->dy_lo}, ymax = {p->y_max_hi, p->y_max_lo};
    DD dx = {p->dx_hi, p->dx_lo}, xmin = {p->x_min_hi, p->x_min_lo};
    DD cy = dd_sub(ymax, dd_mul_f64(dy, sub_j, cpu));
    DD cx = dd_add(xmin, dd_mul_f64(dx, sub_i, cpu));
    return dd_sample(cx, cy, p);
}

/* ------------------------------------------------------------------------- */
/* FP64-delta perturbation: cpu_kernels.py:374-602 (CPU) and                  */
/* cuda_kernels.py:422-590 / :594-815 (CUDA, plain and BLA variants).         */
/* ------------------------------------------------------------------------- */
static void c_mul(double ar, double ai, double br, double bi, double* r, double* i) {
    *r = ar * br - ai * bi;
    *i = ar * bi + ai * br;
}

/* Horner series of cpu_kernels.py:206-223 (u = dc / r). */
static void eval_bbsa(const double* c, double ux, double uy, double* zx, double* zy) {
    int eight = 0;
    for (int q = 8; q < 16; q++) eight |= (c[q] != 0.0);
    double tr, ti;
    if (eight) {
        c_mul(ux, uy, c[14], c[15], &tr, &ti);
        for (int t = 6; t >= 0; t--) c_mul(ux, uy, c[2 * t] + tr, c[2 * t + 1] + ti, &tr, &ti);
    } else {
        c_mul(ux, uy, c[6], c[7], &tr, &ti);
        for (int t = 2; t >= 0; t--) c_mul(ux, uy, c[2 * t] + tr, c[2 * t + 1] + ti, &tr, &ti);
    }
    *zx = tr;
    *zy = ti;
}

static Sample glitch_at(int k) {
    Sample o;
    o.s = (float)k;
    o.s64 = (double)k;
    o.k = k;
    o.glitch = 1;
    return o;
}

static Sample rebase_sample_at(const ApFrameParams* p, const ApFrameBuffers* b, double sub_i,
                               double sub_j);

static Sample pert_sample_at(const ApFrameParams* p, const ApFrameBuffers* b, double sub_i,
                             double sub_j) {
    if (p->flags & AP_FLAG_REBASE) return rebase_sample_at(p, b, sub_i, sub_j);
    const int ft = p->fractal_type, cpu = p->arith == AP_ARITH_REF_CPU;
    const int julia = (ft == 2 || ft == 3);
    const int ref_len = p->ref_len, max_iter = p->max_iter;
    const double* re = b->ref_re;
    const double* im = b->ref_im;
    const int esc_glitch = (p->flags & AP_FLAG_ESCAPE_GLITCH) != 0;
    const int nan_guard = (p->flags & AP_FLAG_NAN_GUARD) != 0;
    const int strict = p->strict_glitch > 0;
    const double dcy = (p->ref_py - sub_j) * p->dy_hi;
    const double dcx = (sub_i - p->ref_px) * p->dx_hi;
    double dzx, dzy;
    int k;
    if (p->bbsa_skip > 0 && (ft == 0 || ft == 2 || ft == 4) &&
        (dcx * p->bbsa_inv_r) * (dcx * p->bbsa_inv_r) + (dcy * p->bbsa_inv_r) * (dcy * p->bbsa_inv_r) <= 1.0) {
        eval_bbsa(p->bbsa, dcx * p->bbsa_inv_r, dcy * p->bbsa_inv_r, &dzx, &dzy);
        k = p->bbsa_skip;
    } else {
        dzx = julia ? dcx : 0.0;
        dzy = julia ? dcy : 0.0;
        k = 0;
    }
    const double dcpx = julia ? 0.0 : dcx, dcpy = julia ? 0.0 : dcy;
    int glitch = 0;
    const int levels = p->bla_levels;
    const int has_bla = levels > 1 && b->bla != NULL && (ft == 0 || ft == 2 || ft == 4);
    const double inv_ln = inv_ln_for(ft, p->gen_n);
    const size_t L = (size_t)ref_len;

    while (k < ref_len) {
        const double rx = re[k], ry = im[k];
        const double zx = rx + dzx, zy = ry + dzy;
        const double mag2 = zx * zx + zy * zy;
        if (mag2 > BAILOUT) {
            if (esc_glitch && strict && k > 15 && (rx * rx + ry * ry) < 4.0) glitch = 1;
            Sample o = escaped(k, mag2, inv_ln);
            o.glitch = glitch;
            return o;
        }
        if (strict && k > 15) {
            const double r_mag2 = rx * rx + ry * ry;
            if (mag2 < 1e-6 * r_mag2 && r_mag2 > 1e-8) glitch = 1;
        }
        if (has_bla && k < ref_len - 1) {
            const double dz_mag2 = dzx * dzx + dzy * dzy;
            if (dz_mag2 < b->bla[((size_t)0 * L + k) * 5 + 4]) {
                int best = 0, max_d = levels - 1;
                if (dz_mag2 == 0.0 && (dzx != 0.0 || dzy != 0.0)) max_d = max_d > 8 ? 8 : max_d;
                for (int d = max_d; d > 0; d--) {
                    if (k + (1 << d) < ref_len && dz_mag2 < b->bla[((size_t)d * L + k) * 5 + 4]) {
                        best = d;
                        break;
                    }
                }
                const double* e = b->bla + ((size_t)best * L + k) * 5;
                const double ar = e[0], ai = e[1], br = e[2], bi = e[3];
                double nx, ny;
                if (cpu) {
                    nx = (ar * dzx - ai * dzy) + (br * dcpx - bi * dcpy);
                    ny = (ar * dzy + ai * dzx) + (br * dcpy + bi * dcpx);
                } else {
                    nx = fma(ar, dzx, fma(-ai, dzy, fma(br, dcpx, -bi * dcpy)));
                    ny = fma(ar, dzy, fma(ai, dzx, fma(br, dcpy, bi * dcpx)));
                }
                dzx = nx;
                dzy = ny;
                if (isnan(dzx) || isnan(dzy) || isinf(dzx) || isinf(dzy)) return glitch_at(k);
                k += 1 << best;
                continue;
            }
        }
        if (ft == 0 || ft == 2) {
            double nx, ny;
            if (cpu) {
                nx = (2.0 * rx + dzx) * dzx - (2.0 * ry + dzy) * dzy + dcpx;
                ny = 2.0 * ((rx + dzx) * dzy + ry * dzx) + dcpy;
            } else {
                nx = fma(2.0 * rx + dzx, dzx, fma(-(2.0 * ry + dzy), dzy, dcpx));
                ny = fma(2.0, fma(rx + dzx, dzy, ry * dzx), dcpy);
            }
            dzx = nx;
            dzy = ny;
        } else if (ft == 1 || ft == 3) {
            const double nx = (2.0 * rx + dzx) * dzx - (2.0 * ry + dzy) * dzy + dcpx;
            const double sx = rx >= 0.0 ? 1.0 : -1.0, sy = ry >= 0.0 ? 1.0 : -1.0;
            const double ddx = (rx + dzx) * sx >= 0.0 ? sx * dzx : -sx * (2.0 * rx + dzx);
            const double ddy = (ry + dzy) * sy >= 0.0 ? sy * dzy : -sy * (2.0 * ry + dzy);
            dzy = 2.0 * (fabs(rx) * ddy + fabs(ry) * ddx + ddx * ddy) - dcpy;
            dzx = nx;
        } else {
            double pr = dzx, pi = dzy, qr = rx, qi = ry;
            for (int t = 0; t < p->gen_n - 1; t++) {
                double t1r, t1i, t2r, t2i;
                c_mul(pr, pi, rx, ry, &t1r, &t1i);
                c_mul(pr + qr, pi + qi, dzx, dzy, &t2r, &t2i);
                pr = t1r + t2r;
                pi = t1i + t2i;
                c_mul(qr, qi, rx, ry, &qr, &qi);
            }
            double kr, ki;
            c_mul(p->gen_kr, p->gen_ki, dzx, dzy, &kr, &ki);
            dzx = pr + kr + dcpx;
            dzy = pi + ki + dcpy;
        }
        k++;
    }

    /* Stage 2: the reference escaped (or the orbit ended); iterate z directly. */
    double zx = re[ref_len] + dzx, zy = im[ref_len] + dzy;
    const double cx = julia ? p->julia_cx_hi : p->ref_cx + dcx;
    const double cy = julia ? p->julia_cy_hi : p->ref_cy + dcy;
    if (ref_len < max_iter) glitch = 1;
    while (k < max_iter) {
        const double zx2 = zx * zx, zy2 = zy * zy;
        const double mag2 = zx2 + zy2;
        if (nan_guard && (isnan(mag2) || isinf(mag2))) return glitch_at(k);
        if (mag2 > BAILOUT) {
            Sample o = escaped(k, mag2, inv_ln);
            o.glitch = glitch;
            return o;
        }
        if (ft == 0 || ft == 2) {
            zy = 2.0 * zx * zy + cy;
            zx = zx2 - zy2 + cx;
        } else if (ft == 1 || ft == 3) {
            zy = 2.0 * fabs(zx) * fabs(zy) - cy;
            zx = zx2 - zy2 + cx;
        } else {
            double zr = zx, zi = zy;
            for (int t = 0; t < p->gen_n - 1; t++) {
                const double nr = zr * zx - zi * zy, ni = zr * zy + zi * zx;
                zr = nr;
                zi = ni;
            }
            const double kzr = p->gen_kr * zx - p->gen_ki * zy;
            const double kzi = p->gen_kr * zy + p->gen_ki * zx;
            zx = zr + kzr + cx;
            zy = zi + kzi + cy;
        }
        k++;
    }
    Sample o = interior();
    o.glitch = glitch;
    return o;
}

/* ------------------------------------------------------------------------- */
/* One-pass rebasing (AP_FLAG_REBASE).  The reference has no such sample: it   */
/* rebases by re-rendering glitched pixels around new references              */
/* (engine.py:1890-2113).  This restates the engine's extension, Zhuoran's    */
/* rebasing (fractalforums.org 2021), in the operation order of the FP64-delta */
/* sample above; its values are pinned by the 700-bit ground truth            */
/* (tests/golden/truth_cfg3.npz) rather than by reference output.             */
/*   k counts the pixel's iterations, m indexes the reference (Z_0 = 0).      */
/*   Each step: z = Z_m + dz; escape when |z|^2 > 65536 (NaN: glitch);        */
/*   when |z|^2 < |dz|^2, or m == ref_len > 0: dz <- z, m <- 0;               */
/*   else the largest BLA level with m + 2^d < ref_len, k + 2^d <= max_iter   */
/*   and |dz|^2 < r_d^2 (levels 0..8 only for an underflowed |dz|^2);         */
/*   else one perturbation step.  Interior after max_iter.                    */
/*   AP_ARITH_FAST (this form only): |dz|^2, |z|^2 as fma(x, x, y*y); the     */
/*   Mandelbrot step a = fma(2, Z, dz), dz' = fma(a, dz, ...) + dc fused; the  */
/*   Burning Ship and Multibrot steps with their products fused into the sums */
/*   (as written below); leaps in the CUDA profile's form.                    */
/* ------------------------------------------------------------------------- */
static int floor_log2(int v) {
    int r = 0;
    while (v > 1) {
        v >>= 1;
        r++;
    }
    return r;
}

static Sample rebase_sample_at(const ApFrameParams* p, const ApFrameBuffers* b, double sub_i,
                               double sub_j) {
    const int ft = p->fractal_type, cpu = p->arith == AP_ARITH_REF_CPU;
    const int fast = p->arith == AP_ARITH_FAST;
    const int ref_len = p->ref_len, max_iter = p->max_iter;
    const double* re = b->ref_re;
    const double* im = b->ref_im;
    const double dcy = (p->ref_py - sub_j) * p->dy_hi;
    const double dcx = (sub_i - p->ref_px) * p->dx_hi;
    double dzx = 0.0, dzy = 0.0;
    int k = 0;
    if (p->bbsa_skip > 0 && (ft == 0 || ft == 4) &&
        (dcx * p->bbsa_inv_r) * (dcx * p->bbsa_inv_r) + (dcy * p->bbsa_inv_r) * (dcy * p->bbsa_inv_r) <= 1.0) {
        eval_bbsa(p->bbsa, dcx * p->bbsa_inv_r, dcy * p->bbsa_inv_r, &dzx, &dzy);
        k = p->bbsa_skip;
    }
    int m = k;
    const int levels = p->bla_levels;
    const int has_bla = levels > 1 && b->bla != NULL && (ft == 0 || ft == 4);
    const double inv_ln = inv_ln_for(ft, p->gen_n);
    const size_t L = (size_t)ref_len;
    while (k < max_iter) {
        const double rx = re[m], ry = im[m];
        const double zx = rx + dzx, zy = ry + dzy;
        const double mag2 = fast ? fma(zx, zx, zy * zy) : zx * zx + zy * zy;
        if (!(mag2 <= BAILOUT)) {
            if (isnan(mag2)) return glitch_at(k);
            return escaped(k, mag2, inv_ln);
        }
        const double dz_mag2 = fast ? fma(dzx, dzx, dzy * dzy) : dzx * dzx + dzy * dzy;
        if (mag2 < dz_mag2 || (m == ref_len && m > 0)) {
            dzx = zx;
            dzy = zy;
            m = 0;
            continue;
        }
        if (has_bla && m < ref_len - 1 && dz_mag2 < b->bla[(size_t)m * 5 + 4]) {
            int best = 0, max_d = levels - 1;
            if (dz_mag2 == 0.0 && (dzx != 0.0 || dzy != 0.0)) max_d = max_d > 8 ? 8 : max_d;
            const int cap = floor_log2(max_iter - k);
            if (max_d > cap) max_d = cap;
            for (int d = max_d; d > 0; d--) {
                if (m + (1 << d) < ref_len && dz_mag2 < b->bla[((size_t)d * L + m) * 5 + 4]) {
                    best = d;
                    break;
                }
            }
            const double* e = b->bla + ((size_t)best * L + m) * 5;
            const double ar = e[0], ai = e[1], br = e[2], bi = e[3];
            double nx, ny;
            if (cpu) {
                nx = (ar * dzx - ai * dzy) + (br * dcx - bi * dcy);
                ny = (ar * dzy + ai * dzx) + (br * dcy + bi * dcx);
            } else {
                nx = fma(ar, dzx, fma(-ai, dzy, fma(br, dcx, -bi * dcy)));
                ny = fma(ar, dzy, fma(ai, dzx, fma(br, dcy, bi * dcx)));
            }
            dzx = nx;
            dzy = ny;
            if (isnan(dzx) || isnan(dzy) || isinf(dzx) || isinf(dzy)) return glitch_at(k);
            m += 1 << best;
            k += 1 << best;
            continue;
        }
        if (ft == 0) {
            double nx, ny;
            if (fast) { /* a = 2Z + dz rounded once; (a dz) + dc fused */
                const double ax = fma(2.0, rx, dzx), ay = fma(2.0, ry, dzy);
                nx = fma(ax, dzx, fma(-ay, dzy, dcx));
                ny = fma(ax, dzy, fma(ay, dzx, dcy));
            } else if (cpu) {
                nx = (2.0 * rx + dzx) * dzx - (2.0 * ry + dzy) * dzy + dcx;
                ny = 2.0 * ((rx + dzx) * dzy + ry * dzx) + dcy;
            } else {
                nx = fma(2.0 * rx + dzx, dzx, fma(-(2.0 * ry + dzy), dzy, dcx));
                ny = fma(2.0, fma(rx + dzx, dzy, ry * dzx), dcy);
            }
            dzx = nx;
            dzy = ny;
        } else if (ft == 1) {
            const double sx = rx >= 0.0 ? 1.0 : -1.0, sy = ry >= 0.0 ? 1.0 : -1.0;
            if (fast) { /* 2Z + dz rounded once; products fused into the sums */
                const double ax = fma(2.0, rx, dzx), ay = fma(2.0, ry, dzy);
                const double nx = fma(ax, dzx, fma(-ay, dzy, dcx));
                const double ddx = (rx + dzx) * sx >= 0.0 ? sx * dzx : -sx * ax;
                const double ddy = (ry + dzy) * sy >= 0.0 ? sy * dzy : -sy * ay;
                dzy = fma(2.0, fma(fabs(rx), ddy, fma(fabs(ry), ddx, ddx * ddy)), -dcy);
                dzx = nx;
            } else {
                const double nx = (2.0 * rx + dzx) * dzx - (2.0 * ry + dzy) * dzy + dcx;
                const double ddx = (rx + dzx) * sx >= 0.0 ? sx * dzx : -sx * (2.0 * rx + dzx);
                const double ddy = (ry + dzy) * sy >= 0.0 ? sy * dzy : -sy * (2.0 * ry + dzy);
                dzy = 2.0 * (fabs(rx) * ddy + fabs(ry) * ddx + ddx * ddy) - dcy;
                dzx = nx;
            }
        } else if (fast) {
            /* (Z + dz)^n - Z^n by P_{j+1} = P_j Z + (P_j + Z^j) dz, each complex product
               sum as one chain of fused multiply-adds, then + k dz + dc */
            double pr = dzx, pi = dzy, qr = rx, qi = ry;
            for (int t = 0; t < p->gen_n - 1; t++) {
                const double sr = pr + qr, si = pi + qi;
                const double npr = fma(pr, rx, fma(-pi, ry, fma(sr, dzx, -si * dzy)));
                const double npi = fma(pr, ry, fma(pi, rx, fma(sr, dzy, si * dzx)));
                const double nqr = fma(qr, rx, -qi * ry), nqi = fma(qr, ry, qi * rx);
                pr = npr;
                pi = npi;
                qr = nqr;
                qi = nqi;
            }
            const double ox = dzx, oy = dzy;
            dzx = fma(p->gen_kr, ox, fma(-p->gen_ki, oy, pr + dcx));
            dzy = fma(p->gen_kr, oy, fma(p->gen_ki, ox, pi + dcy));
        } else {
            double pr = dzx, pi = dzy, qr = rx, qi = ry;
            for (int t = 0; t < p->gen_n - 1; t++) {
                double t1r, t1i, t2r, t2i;
                c_mul(pr, pi, rx, ry, &t1r, &t1i);
                c_mul(pr + qr, pi + qi, dzx, dzy, &t2r, &t2i);
                pr = t1r + t2r;
                pi = t1i + t2i;
                c_mul(qr, qi, rx, ry, &qr, &qi);
            }
            double kr, ki;
            c_mul(p->gen_kr, p->gen_ki, dzx, dzy, &kr, &ki);
            dzx = pr + kr + dcx;
            dzy = pi + ki + dcy;
        }
        m++;
        k++;
    }
    return interior();
}

/* ------------------------------------------------------------------------- */
/* FloatExp tier: cpu_compute_perturbation_sample_floatexp                    */
/* (cpu_kernels.py:606-1021) and compute_perturbation_sample_floatexp[_bla]   */
/* (cuda_kernels.py:819-1499).  The delta is (dzx, dzy) 2^(z_exp - E); the    */
/* pixel offsets are in units of 2^-E.  Every operation is written in source  */
/* order, unfused, except the CUDA BLA leap's explicit fma.                   */
/* ------------------------------------------------------------------------- */
static double pow2_f64(int e) { /* cuda_kernels.py:97-102 */
    if (e >= 1023) return 1.7976931348623157e+308;
    if (e <= -1022) return 0.0;
    return ldexp(1.0, e);
}

static double py_max(double a, double b) { return b > a ? b : a; }

static void renorm16(double* x, double* y, int* e) {
    double mag = py_max(fabs(*x), fabs(*y));
    while (mag > 65536.0 && isfinite(mag)) {
        *x *= 1.52587890625e-05;
        *y *= 1.52587890625e-05;
        *e += 16;
        mag = py_max(fabs(*x), fabs(*y));
    }
    while (mag < 1.52587890625e-05 && mag > 0.0 && isfinite(mag)) {
        *x *= 65536.0;
        *y *= 65536.0;
        *e -= 16;
        mag = py_max(fabs(*x), fabs(*y));
    }
}

/* cpu_kernels.py:171-201 */
static int floatexp_glitch(double rx, double ry, double dzx, double dzy, int eff_exp) {
    const double r_max = py_max(fabs(rx), fabs(ry));
    if (r_max < 1e-4) return 0;
    const double dz_max = py_max(fabs(dzx), fabs(dzy));
    if (dz_max <= 0.0) return 0;
    const int r_exp = (int)(log(r_max) * 1.4426950408889634);
    const int dz_exp = (int)(log(dz_max) * 1.4426950408889634);
    const int diff = r_exp - (eff_exp + dz_exp);
    if (diff > 10 || diff < -10) return 0;
    const double scale_r = pow2_f64(-r_exp), scale_dz = pow2_f64(eff_exp - r_exp);
    const double rxs = rx * scale_r, rys = ry * scale_r;
    const double zx = rxs + dzx * scale_dz, zy = rys + dzy * scale_dz;
    return zx * zx + zy * zy < 1e-6 * (rxs * rxs + rys * rys);
}

static int bla_fits(int scaled, double dz_mag2, double dz_lin, double r_sq) {
    return scaled ? (dz_mag2 < r_sq) : (r_sq > 0.0 && dz_lin < sqrt(r_sq));
}

static Sample floatexp_sample_at(const ApFrameParams* p, const ApFrameBuffers* b, double sub_i,
                                 double sub_j) {
    const int cpu = p->arith == AP_ARITH_REF_CPU;
    const int ft = p->fractal_type;
    const int julia = (ft == 2 || ft == 3);
    const int ref_len = p->ref_len, max_iter = p->max_iter, E = p->e_scale;
    const double* re = b->ref_re;
    const double* im = b->ref_im;
    const int strict = p->strict_glitch > 0;
    const double dcy = (p->ref_py - sub_j) * p->dy_hi;
    const double dcx = (sub_i - p->ref_px) * p->dx_hi;
    double dzx = julia ? dcx : 0.0, dzy = julia ? dcy : 0.0;
    int z_exp = 0, k = 0, glitch = 0;
    const double dcpx = julia ? 0.0 : dcx, dcpy = julia ? 0.0 : dcy;
    const int levels = p->bla_levels;
    const int has_bla = levels > 1 && b->bla != NULL && (ft == 0 || ft == 2 || ft == 4);
    const size_t L = (size_t)ref_len;
    const double inv_ln = inv_ln_for(ft, p->gen_n);

    while (k < ref_len) {
        const double rx = re[k], ry = im[k];
        const int eff_exp = z_exp - E;
        if (eff_exp >= -50) {
            const double sc = pow2_f64(eff_exp);
            const double zx = rx + dzx * sc, zy = ry + dzy * sc;
            const double mag2 = zx * zx + zy * zy;
            if (mag2 > BAILOUT) {
                Sample o = escaped(k, mag2, inv_ln);
                o.glitch = glitch;
                return o;
            }
        }
        if (strict && k > 15 && floatexp_glitch(rx, ry, dzx, dzy, eff_exp)) glitch = 1;

        if (has_bla && k < ref_len - 1) {
            const int scaled = eff_exp >= -510;
            double dz_mag2 = 0.0, dz_lin = 0.0;
            if (scaled) {
                const double sr = pow2_f64(eff_exp);
                dz_mag2 = (dzx * dzx + dzy * dzy) * (sr * sr);
            } else {
                dz_lin = sqrt(dzx * dzx + dzy * dzy) * pow2_f64(eff_exp > -1020 ? eff_exp : -1020);
            }
            if (bla_fits(scaled, dz_mag2, dz_lin, b->bla[(size_t)k * 5 + 4])) {
                int best = 0;
                for (int d = levels - 1; d > 0; d--) {
                    if (k + (1 << d) < ref_len &&
                        bla_fits(scaled, dz_mag2, dz_lin, b->bla[((size_t)d * L + k) * 5 + 4])) {
                        best = d;
                        break;
                    }
                }
                const double* e = b->bla + ((size_t)best * L + k) * 5;
                const double ar = e[0], ai = e[1], br = e[2], bi = e[3];
                const double scale_c = (z_exp >= -1020 && z_exp <= 1020) ? pow2_f64(-z_exp) : 0.0;
                const double cxs = dcpx * scale_c, cys = dcpy * scale_c;
                double nx, ny;
                if (cpu) {
                    nx = (ar * dzx - ai * dzy) + (br * cxs - bi * cys);
                    ny = (ar * dzy + ai * dzx) + (br * cys + bi * cxs);
                } else {
                    nx = fma(ar, dzx, fma(-ai, dzy, fma(br, cxs, -bi * cys)));
                    ny = fma(ar, dzy, fma(ai, dzx, fma(br, cys, bi * cxs)));
                }
                dzx = nx;
                dzy = ny;
                if (isnan(dzx) || isnan(dzy) || isinf(dzx) || isinf(dzy)) return glitch_at(k);
                renorm16(&dzx, &dzy, &z_exp);
                k += 1 << best;
                continue;
            }
        }

        const int shift_nl = z_exp - E;
        const double scale_c = (z_exp >= -1020 && z_exp <= 1020) ? pow2_f64(-z_exp) : 0.0;
        if (ft == 0 || ft == 2) {
            double lx = 2.0 * (rx * dzx - ry * dzy);
            double ly = 2.0 * (rx * dzy + ry * dzx);
            if (shift_nl >= -1020) {
                const double sn = pow2_f64(shift_nl);
                lx += (dzx * dzx - dzy * dzy) * sn;
                ly += (2.0 * dzx * dzy) * sn;
            }
            dzx = lx + dcpx * scale_c;
            dzy = ly + dcpy * scale_c;
        } else if (ft == 1 || ft == 3) {
            const double sn = shift_nl >= -1020 ? pow2_f64(shift_nl) : 0.0;
            const double sx = rx >= 0.0 ? 1.0 : -1.0, sy = ry >= 0.0 ? 1.0 : -1.0;
            if (cpu) { /* cpu_kernels.py:795-829 */
                const double se = eff_exp >= -1020 ? pow2_f64(eff_exp) : 0.0;
                const double inv = eff_exp <= 1020 ? pow2_f64(-eff_exp) : 0.0;
                double fx, ex, fy, ey;
                if ((rx + dzx * se) * sx >= 0.0) { fx = sx; ex = 0.0; }
                else { fx = -sx; ex = eff_exp <= 1020 ? ((-sx * 2.0) * rx) * inv : 0.0; }
                if ((ry + dzy * se) * sy >= 0.0) { fy = sy; ey = 0.0; }
                else { fy = -sy; ey = eff_exp <= 1020 ? ((-sy * 2.0) * ry) * inv : 0.0; }
                const double lx = (2.0 * rx + dzx * sn) * dzx - (2.0 * ry + dzy * sn) * dzy + dcpx * scale_c;
                const double dxn = fx * dzx + ex, dyn = fy * dzy + ey;
                const double ly = 2.0 * (fabs(rx) * dyn + fabs(ry) * dxn + dxn * dyn * sn) - dcpy * scale_c;
                dzx = lx;
                dzy = ly;
            } else { /* cuda_kernels.py:964-985 */
                const double sd = eff_exp >= -60 ? pow2_f64(eff_exp) : 0.0;
                const double inv = pow2_f64(-eff_exp);
                const double ddx = (rx + dzx * sd) * sx >= 0.0 ? sx * dzx : -sx * (2.0 * rx * inv + dzx);
                const double ddy = (ry + dzy * sd) * sy >= 0.0 ? sy * dzy : -sy * (2.0 * ry * inv + dzy);
                double lx = 2.0 * (rx * dzx - ry * dzy);
                double ly = 2.0 * (fabs(rx) * ddy + fabs(ry) * ddx);
                if (shift_nl >= -1020) {
                    lx += (dzx * dzx - dzy * dzy) * sn;
                    ly += (2.0 * ddx * ddy) * sn;
                }
                dzx = lx + dcpx * scale_c;
                dzy = ly - dcpy * scale_c;
            }
        } else {
            const double sn = shift_nl >= -1020 ? pow2_f64(shift_nl) : 0.0;
            double pr = dzx, pi = dzy, qr = rx, qi = ry;
            for (int t = 0; t < p->gen_n - 1; t++) {
                double t1r, t1i, t2r, t2i, t3r, t3i;
                c_mul(pr, pi, rx, ry, &t1r, &t1i);
                c_mul(qr, qi, dzx, dzy, &t2r, &t2i);
                c_mul(pr, pi, dzx, dzy, &t3r, &t3i);
                pr = t1r + t2r + t3r * sn;
                pi = t1i + t2i + t3i * sn;
                c_mul(qr, qi, rx, ry, &qr, &qi);
            }
            double kr, ki;
            c_mul(p->gen_kr, p->gen_ki, dzx, dzy, &kr, &ki);
            dzx = pr + kr + dcpx * scale_c;
            dzy = pi + ki + dcpy * scale_c;
        }
        renorm16(&dzx, &dzy, &z_exp);
        k++;
    }

    /* Stage 2 (cpu_kernels.py:948-1018) */
    const int eff_exp = z_exp - E;
    const double sfb = eff_exp >= -60 ? pow2_f64(eff_exp) : 0.0;
    double zx = re[ref_len] + dzx * sfb, zy = im[ref_len] + dzy * sfb;
    const double scf = E <= 1020 ? pow2_f64(-E) : 0.0;
    const double cx = julia ? p->julia_cx_hi : p->ref_cx + dcpx * scf;
    const double cy = julia ? p->julia_cy_hi : p->ref_cy + dcpy * scf;
    {
        const double mag2 = zx * zx + zy * zy;
        if (mag2 > BAILOUT) {
            Sample o = escaped(ref_len, mag2, inv_ln);
            o.glitch = glitch;
            return o;
        }
    }
    if (ref_len < max_iter) glitch = 1;
    const int nan_guard = (p->flags & AP_FLAG_NAN_GUARD) != 0;
    while (k < max_iter) {
        const double zx2 = zx * zx, zy2 = zy * zy;
        const double mag2 = zx2 + zy2;
        if (nan_guard && (isnan(mag2) || isinf(mag2))) return glitch_at(k);
        if (mag2 > BAILOUT) {
            Sample o = escaped(k, mag2, inv_ln);
            o.glitch = glitch;
            return o;
        }
        if (ft == 0 || ft == 2) {
            zy = 2.0 * zx * zy + cy;
            zx = zx2 - zy2 + cx;
        } else if (ft == 1 || ft == 3) {
            zy = 2.0 * fabs(zx) * fabs(zy) - cy;
            zx = zx2 - zy2 + cx;
        } else {
            double zr = zx, zi = zy;
            for (int t = 0; t < p->gen_n - 1; t++) {
                const double nr = zr * zx - zi * zy, ni = zr * zy + zi * zx;
                zr = nr;
                zi = ni;
            }
            const double kzr = p->gen_kr * zx - p->gen_ki * zy;
            const double kzi = p->gen_kr * zy + p->gen_ki * zx;
            zx = zr + kzr + cx;
            zy = zi + kzi + cy;
        }
        k++;
    }
    Sample o = interior();
    o.glitch = glitch;
    return o;
}

/* ------------------------------------------------------------------------- */
/* FP32-mantissa FloatExp form (AP_TIER_FLOATEXP32).  The engine's own form,  */
/* with no counterpart in the reference: restated here from its definition so */
/* that device frames can be compared with it bit for bit.                    */
/*                                                                            */
/* The delta is w 2^e, w a complex float32 renormalised so that               */
/* max(|w_re|, |w_im|) is in [1, 2) whenever it leaves [2^-16, 2^16];          */
/* delta_c = dcm 2^-E with dcm = (float) of the pixel offset in units of 2^-E.*/
/* A step is evaluated in float32 (products rounded one by one, fmaf where the */
/* form fuses) from the float copy of Z, with S = 2^e and D = dcm 2^(-E-e) as */
/* floats; it is evaluated in FP64 on the FP64 orbit value instead where Z is  */
/* a close approach (|Z|^2 < 2^-100) or the dc term's scale exceeds 2^120.     */
/* Tests on z = Z + dz (escape, Pauldelbrot, one-pass rebasing, Burning Ship's */
/* sign of each component) are decided in FP64 at the steps where a float    */
/* screen says they can fire; the screens are part of the form.  Leaps use    */
/* the chained-BLA table with each coefficient split into a float mantissa    */
/* pair and an exponent, and radii compared as r^2 2^600.                     */
/* ------------------------------------------------------------------------- */
static float fe_exp2i_f(int n) { /* 2^n as float: 0 below 2^-126, 2^127 above */
    if (n > 127) n = 127;
    if (n < -126) return 0.0f;
    union { uint32_t u; float f; } v;
    v.u = (uint32_t)(n + 127) << 23;
    return v.f;
}

static double fe_exp2i_d(int n) { /* 2^n as double: 0 below 2^-1022, inf above 2^1023 */
    if (n < -1022) return 0.0;
    if (n > 1023) return INFINITY;
    union { uint64_t u; double d; } v;
    v.u = (uint64_t)(n + 1023) << 52;
    return v.d;
}

static int fe_ilogb_max(float x, float y) { /* biased exponent field of max(|x|, |y|), minus 127 */
    union { float f; uint32_t u; } v;
    v.f = fmaxf(fabsf(x), fabsf(y));
    return (int)((v.u >> 23) & 0xff) - 127;
}

/* A double pair as one float mantissa pair (larger component in [1, 2)) and an exponent. */
static void fe_split(double re, double im, float* mr, float* mi, int* e) {
    const double m = fmax(fabs(re), fabs(im));
    if (!(m > 0.0) || !isfinite(m)) {
        *mr = *mi = 0.0f;
        *e = 0;
        return;
    }
    union { double d; uint64_t u; } v;
    v.d = m;
    int ex = (int)((v.u >> 52) & 0x7ff) - 1023;
    if (ex < -1022) ex = ilogb(m);
    const double s = ldexp(1.0, -ex);
    *mr = (float)(re * s);
    *mi = (float)(im * s);
    *e = ex;
}

/* (x, y) 2^e renormalised into a float pair; zero and non-finite pairs keep e. */
static void fe_renorm(double x, double y, float* wx, float* wy, int* e) {
    const double m = fmax(fabs(x), fabs(y));
    if (!(m > 0.0) || !isfinite(m)) {
        *wx = (float)x;
        *wy = (float)y;
        return;
    }
    const int ex = ilogb(m);
    const double f = ldexp(1.0, -ex);
    *wx = (float)(x * f);
    *wy = (float)(y * f);
    *e += ex;
}

typedef struct {
    float wx, wy, S, Dx, Dy;
    int e, ec;
    float pdx, pdy;
    double P2;
} FeState;

/* Renormalise w when it is not zero, then refresh S, D and the radius scale 2^(2e + 600). */
static void fe_rescale(FeState* s) {
    if (s->wx != 0.0f || s->wy != 0.0f) {
        const int ex = fe_ilogb_max(s->wx, s->wy);
        if (ex != 0) {
            const float f = fe_exp2i_f(-ex);
            s->wx *= f;
            s->wy *= f;
            s->e += ex;
        }
    }
    s->S = fe_exp2i_f(s->e);
    const float dsc = fe_exp2i_f(s->ec - s->e);
    s->Dx = s->pdx * dsc;
    s->Dy = s->pdy * dsc;
    s->P2 = fe_exp2i_d(2 * s->e + 600);
}

/* The FP64 step of the slow path, in units of 2^e; (cx, cy) the dc term in those units. */
static void fe_step_fp64(const ApFrameParams* p, int form, double Zx, double Zy, double x, double y, int e,
                         double cx, double cy, double* nx, double* ny) {
    const double se = ldexp(1.0, e);
    if (form == 0) {
        *nx = 2.0 * (Zx * x - Zy * y) + se * (x - y) * (x + y) + cx;
        *ny = 2.0 * (Zx * y + Zy * x) + se * 2.0 * x * y + cy;
    } else if (form == 1) {
        const double sx = Zx >= 0.0 ? 1.0 : -1.0, sy = Zy >= 0.0 ? 1.0 : -1.0;
        const double ddx = (Zx + x * se) * sx >= 0.0 ? sx * x : -sx * (ldexp(2.0 * Zx, -e) + x);
        const double ddy = (Zy + y * se) * sy >= 0.0 ? sy * y : -sy * (ldexp(2.0 * Zy, -e) + y);
        *nx = 2.0 * (Zx * x - Zy * y) + se * (x - y) * (x + y) + cx;
        *ny = 2.0 * (fabs(Zx) * ddy + fabs(Zy) * ddx + se * ddx * ddy) - cy;
    } else {
        double pr = x, pi = y, qr = Zx, qi = Zy;
        for (int t = 0; t < p->gen_n - 1; t++) {
            const double sr = se * pr + qr, si = se * pi + qi;
            const double npr = (pr * Zx - pi * Zy) + (sr * x - si * y);
            const double npi = (pr * Zy + pi * Zx) + (sr * y + si * x);
            const double nqr = qr * Zx - qi * Zy, nqi = qr * Zy + qi * Zx;
            pr = npr;
            pi = npi;
            qr = nqr;
            qi = nqi;
        }
        *nx = pr + (p->gen_kr * x - p->gen_ki * y) + cx;
        *ny = pi + (p->gen_kr * y + p->gen_ki * x) + cy;
    }
}

/* The float32 step: Zf the float copy of the orbit value, (Zx, Zy) the FP64 one (read
 * by Burning Ship's sign test where |dz_x| >= |Z_x| / 2 in float). */
static void fe_step_f32(const ApFrameParams* p, int form, float Zfx, float Zfy, double Zx, double Zy,
                        FeState* s, float kr, float ki) {
    const float wx = s->wx, wy = s->wy, S = s->S;
    if (form == 0) {
        const float tx = fmaf(Zfx, wx, -Zfy * wy);
        const float ty = fmaf(Zfx, wy, Zfy * wx);
        const float sq_x = (wx - wy) * (wx + wy);
        const float sq_y = 2.0f * wx * wy;
        s->wx = fmaf(2.0f, tx, fmaf(S, sq_x, s->Dx));
        s->wy = fmaf(2.0f, ty, fmaf(S, sq_y, s->Dy));
    } else if (form == 1) {
        const float sx = Zfx >= 0.0f ? 1.0f : -1.0f, sy = Zfy >= 0.0f ? 1.0f : -1.0f;
        float ddx = sx * wx, ddy = sy * wy;
        const int ux = !(fabsf(wx * S) < 0.5f * fabsf(Zfx));
        const int uy = !(fabsf(wy * S) < 0.5f * fabsf(Zfy));
        const double se = ldexp(1.0, s->e);
        if (ux) {
            const double x = wx, g = Zx >= 0.0 ? 1.0 : -1.0;
            ddx = (Zx + x * se) * g >= 0.0 ? (float)(g * x) : (float)(-g * (ldexp(2.0 * Zx, -s->e) + x));
        }
        if (uy) {
            const double y = wy, g = Zy >= 0.0 ? 1.0 : -1.0;
            ddy = (Zy + y * se) * g >= 0.0 ? (float)(g * y) : (float)(-g * (ldexp(2.0 * Zy, -s->e) + y));
        }
        s->wx = fmaf(2.0f, fmaf(Zfx, wx, -Zfy * wy), fmaf(S, (wx - wy) * (wx + wy), s->Dx));
        s->wy = fmaf(2.0f, fmaf(fabsf(Zfx), ddy, fmaf(fabsf(Zfy), ddx, S * (ddx * ddy))), -s->Dy);
    } else {
        float pr = wx, pi = wy, qr = Zfx, qi = Zfy;
        for (int t = 0; t < p->gen_n - 1; t++) {
            const float sr = fmaf(S, pr, qr), si = fmaf(S, pi, qi);
            const float npr = fmaf(pr, Zfx, fmaf(-pi, Zfy, fmaf(sr, wx, -si * wy)));
            const float npi = fmaf(pr, Zfy, fmaf(pi, Zfx, fmaf(sr, wy, si * wx)));
            const float nqr = fmaf(qr, Zfx, -qi * Zfy), nqi = fmaf(qr, Zfy, qi * Zfx);
            pr = npr;
            pi = npi;
            qr = nqr;
            qi = nqi;
        }
        s->wx = fmaf(kr, wx, fmaf(-ki, wy, pr + s->Dx));
        s->wy = fmaf(kr, wy, fmaf(ki, wx, pi + s->Dy));
    }
}

/* Stage 2's direct FP64 step z <- f(z) + c. */
static void fe_direct_step(const ApFrameParams* p, int form, double* zx, double* zy, double zx2, double zy2,
                           double cx, double cy) {
    if (form == 0) {
        *zy = 2.0 * *zx * *zy + cy;
        *zx = zx2 - zy2 + cx;
    } else if (form == 1) {
        *zy = 2.0 * fabs(*zx) * fabs(*zy) - cy;
        *zx = zx2 - zy2 + cx;
    } else {
        double zr = *zx, zi = *zy;
        for (int t = 0; t < p->gen_n - 1; t++) {
            const double nr = zr * *zx - zi * *zy, ni = zr * *zy + zi * *zx;
            zr = nr;
            zi = ni;
        }
        const double kzr = p->gen_kr * *zx - p->gen_ki * *zy;
        const double kzi = p->gen_kr * *zy + p->gen_ki * *zx;
        *zx = zr + kzr + cx;
        *zy = zi + kzi + cy;
    }
}

/* One sample of the FP32 form.  Without AP_FLAG_REBASE: one reference, Pauldelbrot flags
 * (strict_glitch), FP64 direct iteration after the reference ends.  With it (fractal types
 * 0, 1, 4): when |Z_m + dz| < |dz| or the reference has ended, dz <- Z_m + dz and m <- 0. */
static Sample fe32_sample_at(const ApFrameParams* p, const ApFrameBuffers* b, double sub_i, double sub_j) {
    const int ft = p->fractal_type;
    const int form = (ft == 0 || ft == 2) ? 0 : ((ft == 1 || ft == 3) ? 1 : 4);
    const int rebase = (p->flags & AP_FLAG_REBASE) != 0;
    const int bla = p->bla_levels > 1 && b->bla != NULL && form != 1;
    const int ref_len = p->ref_len, max_iter = p->max_iter, levels = p->bla_levels;
    const double* re = b->ref_re;
    const double* im = b->ref_im;
    const double* T = b->bla;
    const size_t L = (size_t)ref_len;
    const double dcy_n = (p->ref_py - sub_j) * p->dy_hi;
    const double dcx_n = (sub_i - p->ref_px) * p->dx_hi;
    const int julia = ft == 2 || ft == 3;
    const float dcmx = (float)dcx_n, dcmy = (float)dcy_n;
    const float kr = (float)p->gen_kr, ki = (float)p->gen_ki;
    FeState s;
    s.ec = -p->e_scale;
    s.e = s.ec;
    s.pdx = julia ? 0.0f : dcmx;
    s.pdy = julia ? 0.0f : dcmy;
    s.wx = julia ? dcmx : 0.0f;
    s.wy = julia ? dcmy : 0.0f;
    fe_rescale(&s);
    const int strict = !rebase && p->strict_glitch > 0;
    const double inv_ln = inv_ln_for(ft, p->gen_n);
    int k = 0, lim = max_iter, glitch = 0;
    while (rebase ? (k < lim) : (k < ref_len)) {
        const double Zx = re[k], Zy = im[k];
        const double r2 = Zx * Zx + Zy * Zy;
        const float Zfx = (float)Zx, Zfy = (float)Zy, Zfr2 = (float)r2;
        const int close = r2 < 0x1p-100;
        const float wm2 = s.wx * s.wx + s.wy * s.wy;
        if (rebase) {
            int test = k == ref_len || close || (s.e >= -53 && wm2 * (s.S * s.S) > 0.2f * Zfr2);
            if (!test && s.e >= -40) {
                const float zx = Zfx + s.wx * s.S, zy = Zfy + s.wy * s.S;
                test = zx * zx + zy * zy > 65535.0f;
            }
            if (test) {
                const double sc = ldexp(1.0, s.e), x = s.wx, y = s.wy;
                const double ax = Zx + x * sc, ay = Zy + y * sc;
                const double mag2 = ax * ax + ay * ay;
                if (!(mag2 <= BAILOUT)) {
                    const int kk = k + (max_iter - lim);
                    if (isnan(mag2)) return glitch_at(kk);
                    return escaped(kk, mag2, inv_ln);
                }
                double bx = ldexp(Zx, -s.e) + x, by = ldexp(Zy, -s.e) + y;
                if ((k == ref_len && k > 0) || bx * bx + by * by < x * x + y * y) {
                    if (!(fabs(bx) + fabs(by) < 1e300)) {
                        bx = ax;
                        by = ay;
                        s.e = 0;
                    }
                    fe_renorm(bx, by, &s.wx, &s.wy, &s.e);
                    fe_rescale(&s);
                    lim -= k;
                    k = 0;
                    continue;
                }
            }
        } else if (s.e >= -40 || (strict && k > 15 && s.e >= -75)) {
            const float zx = Zfx + s.wx * s.S, zy = Zfy + s.wy * s.S;
            const float zm2 = zx * zx + zy * zy;
            const int near_escape = s.e >= -40 && zm2 > 65535.0f;
            const int near_glitch = strict && k > 15 && zm2 < 2e-6f * Zfr2;
            if (near_escape || near_glitch) {
                const double sc = ldexp(1.0, s.e);
                const double ax = Zx + (double)s.wx * sc, ay = Zy + (double)s.wy * sc;
                const double mag2 = ax * ax + ay * ay;
                if (mag2 > BAILOUT) {
                    Sample o = escaped(k, mag2, inv_ln);
                    o.glitch = glitch;
                    return o;
                }
                if (near_glitch) {
                    const double thr = r2 > 1e-8 ? 1e-6 * r2 : -1.0;
                    if (mag2 < thr) glitch = 1;
                }
            }
        }
        if (bla && k < ref_len - 1) {
            const double dzs = (double)wm2 * s.P2;
#define FE_RADIUS(d) ((d) < levels ? ldexp(T[((size_t)(d) * L + k) * 5 + 4], 600) : 0.0)
            if (dzs < FE_RADIUS(0)) {
                int lo = 0, hi = levels - 1;
                if (rebase) {
                    const int cap = 31 - __builtin_clz((unsigned)(lim - k));
                    if (hi > cap) hi = cap;
                }
                for (int it = 0; it < 4; it++) {
                    if (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (dzs < FE_RADIUS(mid)) lo = mid;
                        else hi = mid - 1;
                    }
                }
                const double* c = T + ((size_t)lo * L + k) * 5;
                float ar, ai, br, bi;
                int ea, eb;
                fe_split(c[0], c[1], &ar, &ai, &ea);
                fe_split(c[2], c[3], &br, &bi, &eb);
                const int fe = eb + s.ec - s.e - ea;
                if (fe >= -120 && fe <= 120) {
                    const float f = fe_exp2i_f(fe);
                    const float bx = (br * s.pdx - bi * s.pdy) * f;
                    const float by = (br * s.pdy + bi * s.pdx) * f;
                    const float nx = fmaf(ar, s.wx, fmaf(-ai, s.wy, bx));
                    const float ny = fmaf(ar, s.wy, fmaf(ai, s.wx, by));
                    s.wx = nx;
                    s.wy = ny;
                    s.e += ea;
                } else {
                    const double bx = ldexp((double)br * s.pdx - (double)bi * s.pdy, fe);
                    const double by = ldexp((double)br * s.pdy + (double)bi * s.pdx, fe);
                    const double nx = (double)ar * s.wx - (double)ai * s.wy + bx;
                    const double ny = (double)ar * s.wy + (double)ai * s.wx + by;
                    s.e += ea;
                    fe_renorm(nx, ny, &s.wx, &s.wy, &s.e);
                }
                fe_rescale(&s);
                k += 1 << lo;
                continue;
            }
#undef FE_RADIUS
        }
        if (close || s.ec - s.e > 120) {
            double nx, ny;
            fe_step_fp64(p, form, Zx, Zy, s.wx, s.wy, s.e, ldexp((double)s.pdx, s.ec - s.e),
                         ldexp((double)s.pdy, s.ec - s.e), &nx, &ny);
            fe_renorm(nx, ny, &s.wx, &s.wy, &s.e);
            fe_rescale(&s);
            k++;
            continue;
        }
        fe_step_f32(p, form, Zfx, Zfy, Zx, Zy, &s, kr, ki);
        const float mx = fmaxf(fabsf(s.wx), fabsf(s.wy));
        if (mx > 65536.0f || (mx < 1.52587890625e-05f && mx > 0.0f)) fe_rescale(&s);
        k++;
    }
    if (rebase) return interior();
    /* stage 2: FP64 direct iteration from Z_ref_len + dz, c = ref_c + dc */
    const double sc = ldexp(1.0, s.e);
    double zx = re[ref_len] + (double)s.wx * sc, zy = im[ref_len] + (double)s.wy * sc;
    const double dct_x = dcx_n * ldexp(1.0, s.ec), dct_y = dcy_n * ldexp(1.0, s.ec);
    const double cx = julia ? p->julia_cx_hi : p->ref_cx + dct_x;
    const double cy = julia ? p->julia_cy_hi : p->ref_cy + dct_y;
    if (!(zx * zx + zy * zy > BAILOUT) && ref_len < max_iter) glitch = 1;
    const int nan_guard = (p->flags & AP_FLAG_NAN_GUARD) != 0;
    while (k < max_iter) {
        const double zx2 = zx * zx, zy2 = zy * zy;
        const double mag2 = zx2 + zy2;
        if (nan_guard && (isnan(mag2) || isinf(mag2))) return glitch_at(k);
        if (mag2 > BAILOUT) {
            Sample o = escaped(k, mag2, inv_ln);
            o.glitch = glitch;
            return o;
        }
        fe_direct_step(p, form, &zx, &zy, zx2, zy2, cx, cy);
        k++;
    }
    Sample o = interior();
    o.glitch = glitch;
    return o;
}

/* ------------------------------------------------------------------------- */
/* Chained BLA table: _jit_build_bla_table (high_precision.py:1101-1238).     */
/* The reference builds it with a fastmath Numba kernel; the fused forms      */
/* below are the ones its compiled x86-64 code evaluates.                     */
/* ------------------------------------------------------------------------- */
static int build_bla_impl(const double* re, const double* im, int ref_len, int ft, double tol,
                          double dc_max, int levels, int gen_n, double kr, double ki, double* T) {
    const size_t L = (size_t)ref_len;
    memset(T, 0, sizeof(double) * (size_t)levels * L * 5);
    if (!(ft == 0 || ft == 2 || ft == 4) || ref_len < 4 || tol <= 0.0) return AP_OK;
    const double tol_sq_4 = (tol * tol) * 4.0;
    for (int k = 0; k < ref_len - 1; k++) {
        const double rx = re[k], ry = im[k];
        double* e = T + (size_t)k * 5;
        const double r_mag2 = fma(ry, ry, rx * rx);
        if (ft == 0 || ft == 2) {
            e[0] = 2.0 * rx;
            e[1] = 2.0 * ry;
            e[2] = 1.0;
            e[3] = 0.0;
            double r_sq = tol_sq_4 * r_mag2;
            r_sq = 0.25 < r_sq ? 0.25 : r_sq;
            if (k == 0 && r_mag2 < 1e-14) r_sq = 0.0;
            e[4] = r_sq;
        } else {
            /* Multibrot: A = n R^(n-1) + K, radius from the quadratic bound (high_precision.py:1126-1175). */
            double zr = 1.0, zi = 0.0;
            for (int t = 0; t < gen_n - 1; t++) {
                const double nr = fma(zr, rx, -(zi * ry)), ni = fma(zr, ry, zi * rx);
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
            } else {
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
        }
    }
    int step = 1;
    for (int d = 1; d < levels; d++) {
        const int step_next = step * 2;
        for (int k = 0; k < ref_len - step_next; k++) {
            const double* e1 = T + ((size_t)(d - 1) * L + k) * 5;
            const double* e2 = T + ((size_t)(d - 1) * L + k + step) * 5;
            double* o = T + ((size_t)d * L + k) * 5;
            const double r1 = e1[4], r2 = e2[4];
            if (!(r1 > 0.0 && r2 > 0.0)) continue;
            const double a1r = e1[0], a1i = e1[1], b1r = e1[2], b1i = e1[3];
            const double a2r = e2[0], a2i = e2[1], b2r = e2[2], b2i = e2[3];
            const double ar = fma(a2r, a1r, -(a2i * a1i));
            const double ai = fma(a2i, a1r, a2r * a1i);
            if (dc_max >= 0.0) {
                /* dc-aware merge: the second leap sees |dz1| <= |A1| |dz| + |B1| dcmax. */
                const double br = fma(a2r, b1r, -(a2i * b1i)) + b2r;
                const double bi = fma(a2i, b1r, fma(a2r, b1i, b2i));
                if (fma(ar, ar, ai * ai) > 1e150 || fma(br, br, bi * bi) > 1e150) continue;
                const double a1_mag = sqrt(fma(a1i, a1i, a1r * a1r));
                const double b1_mag = sqrt(fma(b1i, b1i, b1r * b1r));
                double r = sqrt(r1);
                if (a1_mag > 1e-300) {
                    const double r2c = (sqrt(r2) - b1_mag * dc_max) / a1_mag;
                    r = r < r2c ? r : r2c;
                }
                if (!(r > 0.0)) continue;
                o[0] = ar;
                o[1] = ai;
                o[2] = br;
                o[3] = bi;
                o[4] = r * r < r1 ? r * r : r1; /* sqrt then square may round up by an ulp */
                continue;
            }
            const double a_mag2 = fma(ar, ar, ai * ai);
            if (a_mag2 > 1e150) {
                o[0] = o[1] = o[2] = o[3] = o[4] = 0.0;
                continue;
            }
            const double br = fma(a2r, b1r, -(a2i * b1i)) + b2r;
            const double bi = fma(a2i, b1r, fma(a2r, b1i, b2i));
            const double b_mag2 = fma(br, br, bi * bi);
            if (b_mag2 > 1e150) {
                o[0] = o[1] = o[2] = o[3] = o[4] = 0.0;
                continue;
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
        step = step_next;
    }
    return AP_OK;
}

APO_EXPORT int apo_build_bla(const double* re, const double* im, int ref_len, int ft, double tol,
                             int levels, int gen_n, double kr, double ki, double* T) {
    return build_bla_impl(re, im, ref_len, ft, tol, -1.0, levels, gen_n, kr, ki, T);
}

/* Chained BLA with the dc-aware merge of Zhuoran's published method
 * (fractalforums.org, 2021): r = max(0, min(r1, (r2 - |B1| dcmax) / |A1|)).
 * Level 0 is the reference's (high_precision.py:1126-1175) with tol = eps.
 * No counterpart in the reference. */
APO_EXPORT int apo_build_bla_dc(const double* re, const double* im, int ref_len, int ft, double eps,
                                double dc_max, int levels, int gen_n, double kr, double ki, double* T) {
    if (!(dc_max >= 0.0)) return AP_E_INVALID;
    return build_bla_impl(re, im, ref_len, ft, eps, dc_max, levels, gen_n, kr, ki, T);
}

/* ------------------------------------------------------------------------- */
/* Exported oracle entry points (apo_*: host pointers, same structs as ap_*)  */
/* ------------------------------------------------------------------------- */
APO_EXPORT int apo_abi_version(void) { return AP_ABI_VERSION; }

APO_EXPORT int apo_render_pass(const ApFrameParams* p, const ApFrameBuffers* b) {
    if (!p || !b || p->width <= 0 || p->height <= 0 || p->factor < 1) return AP_E_INVALID;
    render_pass(p, b, 0);
    return AP_OK;
}

APO_EXPORT int apo_resolve_hist_pass(const ApFrameParams* p, const ApFrameBuffers* b) {
    if (!p || !b || p->width <= 0 || p->height <= 0 || p->factor < 1) return AP_E_INVALID;
    render_pass(p, b, 1);
    return AP_OK;
}

/* cuda_kernels.py:1587-1611 (float32 difference against the float32 threshold). */
APO_EXPORT int apo_edge_detect(const float* it, uint8_t* edge, int W, int H, float thr) {
    for (int j = 0; j < H; j++) {
        for (int i = 0; i < W; i++) {
            float s = it[(size_t)j * W + i];
            int e = 0;
            for (int dj = -1; dj <= 1 && !e; dj++) {
                int nj = j + dj;
                if (nj < 0 || nj >= H) continue;
                for (int di = -1; di <= 1; di++) {
                    int ni = i + di;
                    if (ni < 0 || ni >= W || (di == 0 && dj == 0)) continue;
                    float sn = it[(size_t)nj * W + ni];
                    float d = s - sn;
                    if ((s < 0.0f) != (sn < 0.0f) || (s >= 0.0f && fabsf(d) > thr)) {
                        e = 1;
                        break;
                    }
                }
            }
            edge[(size_t)j * W + i] = (uint8_t)e;
        }
    }
    return AP_OK;
}

/* cuda_kernels.py:1922-2013: histogram, float64 prefix sum, normalised float32 CDF. */
APO_EXPORT int apo_histogram_cdf(const float* it, int W, int H, int max_iter, int num_bins,
                                 int32_t* hist, float* cdf) {
    memset(hist, 0, sizeof(int32_t) * (size_t)num_bins);
    const double inv_max = 1.0 / fmax(1.0, (double)max_iter);
    for (size_t q = 0; q < (size_t)W * H; q++) {
        float s = it[q];
        if (s >= 0.0f) {
            double pos = ((double)s * inv_max) * (double)(num_bins - 1);
            int bin = (int)pos;
            if (bin >= num_bins) bin = num_bins - 1;
            else if (bin < 0) bin = 0;
            hist[bin] += 1;
        }
    }
    double total = 0.0;
    for (int q = 0; q < num_bins; q++) total += (double)hist[q];
    double run = 0.0;
    for (int q = 0; q < num_bins; q++) {
        run += (double)hist[q];
        cdf[q] = total > 0.0 ? (float)(run / total) : (float)((double)q / (double)(num_bins - 1));
    }
    return AP_OK;
}

/* apply_histogram_equalization_kernel (cuda_kernels.py:2016) and
 * recolor_iter_map_cuda_kernel (cuda_kernels.py:3201). */
static void colour_row(void* vctx, int j) {
    const PassCtx* c = (const PassCtx*)vctx;
    const ApFrameParams* p = c->p;
    const ApFrameBuffers* b = c->b;
    const int hist = p->scheme_id == 11 && b->cdf != NULL;
    for (int i = 0; i < p->width; i++) {
        size_t idx = (size_t)j * p->width + i;
        double s = b->iter_map[idx];
        double r = 0, g = 0, bb = 0;
        if (s >= 0.0) lut_lerp(b->lut, colour_norm(p, b, s, hist), &r, &g, &bb);
        put_rgb(p, b->rgb, idx, r, g, bb);
    }
}

APO_EXPORT int apo_colour(const ApFrameParams* p, const ApFrameBuffers* b) {
    PassCtx c = {p, b, 0};
    parallel_rows(p->height, colour_row, &c);
    return AP_OK;
}

/* ------------------------------------------------------------------------- */
/* Strict Metric fallback on the device: 34 x 32-bit fixed point              */
/* (compute_ml_sample and ml_*, math_core/cuda_kernels.py:2239-2446).         */
/* ------------------------------------------------------------------------- */
#define ML_N AP_STRICT_NLIMBS

static void ml_add_mag(const uint32_t* a, const uint32_t* b, uint32_t* o) {
    uint64_t carry = 0;
    for (int i = ML_N - 1; i >= 0; i--) {
        uint64_t s = (uint64_t)a[i] + (uint64_t)b[i] + carry;
        o[i] = (uint32_t)(s & 0xFFFFFFFFu);
        carry = s >> 32;
    }
}

static void ml_sub_mag(const uint32_t* a, const uint32_t* b, uint32_t* o) {
    int64_t borrow = 0;
    for (int i = ML_N - 1; i >= 0; i--) {
        int64_t diff = (int64_t)a[i] - (int64_t)b[i] - borrow;
        if (diff < 0) {
            diff += 4294967296LL;
            borrow = 1;
        } else {
            borrow = 0;
        }
        o[i] = (uint32_t)(diff & 0xFFFFFFFF);
    }
}

static int ml_cmp_mag(const uint32_t* a, const uint32_t* b) {
    for (int i = 0; i < ML_N; i++) {
        if (a[i] > b[i]) return 1;
        if (a[i] < b[i]) return -1;
    }
    return 0;
}

static int ml_add_signed(int as, const uint32_t* a, int bs, const uint32_t* b, uint32_t* o) {
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

static int ml_sub_signed(int as, const uint32_t* a, int bs, const uint32_t* b, uint32_t* o) {
    return ml_add_signed(as, a, bs == 0 ? 1 : 0, b, o);
}

static void ml_mul_mag(const uint32_t* a, const uint32_t* b, uint32_t* o) {
    uint64_t carry = 0;
    for (int k = ML_N - 1; k >= 0; k--) {
        uint64_t sum = carry;
        for (int i = 0; i <= k; i++) sum += ((uint64_t)a[i] * (uint64_t)b[k - i]) & 0xFFFFFFFFu;
        if (k + 1 < ML_N) {
            for (int i = 0; i <= k + 1; i++) sum += ((uint64_t)a[i] * (uint64_t)b[k + 1 - i]) >> 32;
        } else {
            for (int i = 1; i < ML_N; i++) sum += ((uint64_t)a[i] * (uint64_t)b[ML_N - i]) >> 32;
        }
        o[k] = (uint32_t)(sum & 0xFFFFFFFFu);
        carry = sum >> 32;
    }
}

static float ml_sample(int cxs, const uint32_t* cxl, int cys, const uint32_t* cyl, int max_iter, int ft,
                       int jxs, const uint32_t* jxl, int jys, const uint32_t* jyl) {
    uint32_t zx[ML_N], zy[ML_N], zx2[ML_N], zy2[ML_N], zxy[ML_N], two_zxy[ML_N], sub_xy[ML_N], tmp[ML_N];
    const uint32_t *cx, *cy;
    int zxs = 0, zys = 0, c_xs, c_ys;
    memset(zx, 0, sizeof zx);
    memset(zy, 0, sizeof zy);
    if (ft == 4) return -1.0f;
    if (ft == 2 || ft == 3) {
        memcpy(zx, cxl, sizeof zx);
        memcpy(zy, cyl, sizeof zy);
        zxs = cxs;
        zys = cys;
        c_xs = jxs;
        c_ys = jys;
        cx = jxl;
        cy = jyl;
    } else {
        c_xs = cxs;
        c_ys = cys;
        cx = cxl;
        cy = cyl;
    }
    for (int k = 0; k < max_iter; k++) {
        if (ft == 1 || ft == 3) zxs = zys = 0;
        ml_mul_mag(zx, zx, zx2);
        ml_mul_mag(zy, zy, zy2);
        if (zx2[0] >= 65536u || zy2[0] >= 65536u || (uint64_t)zx2[0] + (uint64_t)zy2[0] >= 65536u) {
            double mag2 = (double)zx2[0] + (double)zy2[0] + ((double)zx2[1] + (double)zy2[1]) * 2.3283064365386963e-10;
            return escaped(k, mag2, INV_LN2).s;
        }
        int zxys = zxs == zys ? 0 : 1;
        ml_mul_mag(zx, zy, zxy);
        ml_add_mag(zxy, zxy, two_zxy);
        int subs = ml_sub_signed(0, zx2, 0, zy2, sub_xy);
        zxs = ml_add_signed(subs, sub_xy, c_xs, cx, tmp);
        memcpy(zx, tmp, sizeof zx);
        if (ft == 1 || ft == 3)
            zys = ml_sub_signed(0, two_zxy, c_ys, cy, tmp);
        else
            zys = ml_add_signed(zxys, two_zxy, c_ys, cy, tmp);
        memcpy(zy, tmp, sizeof zy);
    }
    return -1.0f;
}

/* eval_glitched_pixels_cuda_kernel / _hist_ (math_core/cuda_kernels.py:2450-2569):
   each listed pixel iterated on its own in FP64, double-double or fixed point, then the
   float32 value, its colour (black below 0) and a cleared glitch flag written. */
APO_EXPORT int apo_strict_eval(const ApFrameParams* p, const ApFrameBuffers* b, const ApStrictView* v,
                               const int32_t* coords, const int32_t* signs, const uint32_t* limbs, int n) {
    const int hist = p->scheme_id == 11 && b->cdf != NULL;
    ApFrameParams q = *p;
    q.arith = AP_ARITH_REF_CUDA;
    for (int t = 0; t < n; t++) {
        int r = coords[2 * t], c = coords[2 * t + 1];
        if (r < 0 || r >= p->height || c < 0 || c >= p->width) continue;
        float s;
        if (v->tier == AP_STRICT_DD) {
            s = dd_sample_at(&q, (double)c, (double)r).s;
        } else if (v->tier == AP_STRICT_FP64) { /* precision_tier 0, cuda_kernels.py:2474-2477 */
            const double x = p->x_min_hi + (double)c * p->dx_hi;
            const double y = p->y_max_hi - (double)r * p->dy_hi;
            s = fp64_sample(x, y, &q).s;
        } else {
            const uint32_t* l = limbs + (size_t)t * 2 * ML_N;
            s = ml_sample(signs[2 * t], l, signs[2 * t + 1], l + ML_N, p->max_iter, p->fractal_type,
                          v->jx_sign, v->jx_limbs, v->jy_sign, v->jy_limbs);
        }
        size_t idx = (size_t)r * p->width + c;
        b->iter_map[idx] = s;
        double cr = 0, cg = 0, cb = 0;
        if (s >= 0.0f) lut_lerp(b->lut, colour_norm(p, b, (double)s, hist), &cr, &cg, &cb);
        put_rgb(p, b->rgb, idx, cr, cg, cb);
        if (b->glitch_out) b->glitch_out[idx] = 0;
    }
    return AP_OK;
}

/* Strict Metric write-back (math_core/engine.py:252-266): iter_map = float32 of the
   value, the float64 value's colour unless it is < 0 or >= max_iter (then black),
   glitch flag cleared. */
APO_EXPORT int apo_set_pixels(const ApFrameParams* p, const ApFrameBuffers* b, const int32_t* coords,
                              const double* values, int n) {
    const int hist = p->scheme_id == 11 && b->cdf != NULL;
    for (int q = 0; q < n; q++) {
        int r = coords[2 * q], c = coords[2 * q + 1];
        if (r < 0 || r >= p->height || c < 0 || c >= p->width) continue;
        size_t idx = (size_t)r * p->width + c;
        double s = values[q];
        b->iter_map[idx] = (float)s;
        double cr = 0, cg = 0, cb = 0;
        if (s >= 0.0 && s < (double)p->max_iter) lut_lerp(b->lut, colour_norm(p, b, s, hist), &cr, &cg, &cb);
        put_rgb(p, b->rgb, idx, cr, cg, cb);
        if (b->glitch_out) b->glitch_out[idx] = 0;
    }
    return AP_OK;
}

/* Per-sample FP64 values on an explicit coordinate grid (x per column, y per row). */
typedef struct {
    const ApFrameParams* p;
    const double* xs;
    const double* ys;
    int W;
    float* s32;
    double* s64;
    int32_t* kmap;
} GridCtx;

static void grid_row(void* vctx, int j) {
    const GridCtx* c = (const GridCtx*)vctx;
    for (int i = 0; i < c->W; i++) {
        Sample o = fp64_sample(c->xs[i], c->ys[j], c->p);
        size_t idx = (size_t)j * c->W + i;
        if (c->s32) c->s32[idx] = o.s;
        if (c->s64) c->s64[idx] = o.s64;
        if (c->kmap) c->kmap[idx] = o.k;
    }
}

/* Samples of any tier at sub-sample coordinates (columns xs, rows ys), each mapped as the
 * unified pass maps it (sample_at). */
typedef struct {
    const ApFrameParams* p;
    const ApFrameBuffers* b;
    const double* xs;
    const double* ys;
    int W;
    double* s64;
    int32_t* kmap;
} SampleGridCtx;

static void sample_grid_row(void* vctx, int j) {
    const SampleGridCtx* c = (const SampleGridCtx*)vctx;
    for (int i = 0; i < c->W; i++) {
        Sample o = sample_at(c->p, c->b, c->xs[i], c->ys[j]);
        size_t idx = (size_t)j * c->W + i;
        c->s64[idx] = o.s64;
        c->kmap[idx] = o.k;
    }
}

APO_EXPORT int apo_sample_grid(const ApFrameParams* p, const ApFrameBuffers* b, const double* xs,
                               const double* ys, int W, int H, double* s64, int32_t* kmap) {
    SampleGridCtx c = {p, b, xs, ys, W, s64, kmap};
    parallel_rows(H, sample_grid_row, &c);
    return AP_OK;
}

APO_EXPORT int apo_fp64_grid(const ApFrameParams* p, const double* xs, const double* ys, int W, int H,
                             float* s32, double* s64, int32_t* kmap) {
    GridCtx c = {p, xs, ys, W, s32, s64, kmap};
    parallel_rows(H, grid_row, &c);
    return AP_OK;
}

/* Number of worker threads (0 = all online cores). */
APO_EXPORT void apo_set_threads(int n) { g_threads = n < 0 ? 0 : n; }

/* Per-sample perturbation values at explicit sub-sample coordinates. */
typedef struct {
    const ApFrameParams* p;
    const ApFrameBuffers* b;
    const double* xs;
    const double* ys;
    int W;
    float* s32;
    uint8_t* glitch;
    int32_t* kmap;
} PertGridCtx;

static void pert_grid_row(void* vctx, int j) {
    const PertGridCtx* c = (const PertGridCtx*)vctx;
    for (int i = 0; i < c->W; i++) {
        Sample o = c->p->tier == AP_TIER_FLOATEXP     ? floatexp_sample_at(c->p, c->b, c->xs[i], c->ys[j])
                   : c->p->tier == AP_TIER_FLOATEXP32 ? fe32_sample_at(c->p, c->b, c->xs[i], c->ys[j])
                                                      : pert_sample_at(c->p, c->b, c->xs[i], c->ys[j]);
        size_t idx = (size_t)j * c->W + i;
        c->s32[idx] = o.s;
        if (c->b->s64) c->b->s64[idx] = o.s64;
        c->glitch[idx] = (uint8_t)(o.glitch > 0);
        if (c->kmap) c->kmap[idx] = o.k;
    }
}

APO_EXPORT int apo_pert_grid(const ApFrameParams* p, const ApFrameBuffers* b, const double* xs,
                             const double* ys, int W, int H, float* s32, uint8_t* glitch, int32_t* kmap) {
    PertGridCtx c = {p, b, xs, ys, W, s32, glitch, kmap};
    parallel_rows(H, pert_grid_row, &c);
    return AP_OK;
}
