// ap_colour.cu -- edge mask, histogram -> CDF, and colouring passes.
#include "ap_common.cuh"

namespace ap {

// ------------------------------------------------------------------ edges
// math_core/cuda_kernels.py:1587-1611: a pixel is an edge when any of its
// 8 neighbours differs in interior-ness or by more than the threshold
// (float32 difference against the float32 threshold).
__global__ void __launch_bounds__(256) edge_kernel(const float* __restrict__ it,
                                                   uint8_t* __restrict__ edge, int W, int H,
                                                   float thr) {
    const int i = blockIdx.x * 16 + (threadIdx.x & 15);
    const int j = blockIdx.y * 16 + (threadIdx.x >> 4);
    if (i >= W || j >= H) return;
    const float s = it[(size_t)j * W + i];
    bool e = false;
    for (int dj = -1; dj <= 1 && !e; ++dj) {
        const int nj = j + dj;
        if (nj < 0 || nj >= H) continue;
        for (int di = -1; di <= 1; ++di) {
            const int ni = i + di;
            if (ni < 0 || ni >= W || (di == 0 && dj == 0)) continue;
            const float sn = it[(size_t)nj * W + ni];
            if ((s < 0.0f) != (sn < 0.0f) || (s >= 0.0f && fabsf(__fsub_rn(s, sn)) > thr)) {
                e = true;
                break;
            }
        }
    }
    edge[(size_t)j * W + i] = e ? 1 : 0;
}

// -------------------------------------------------------------- histogram
// math_core/cuda_kernels.py:1999-2013: bin = int(s / max(1, max_iter) * (bins - 1)).
// Neighbouring pixels mostly fall into the same bins, so the lanes of a warp that count
// into one bin add once (the lowest of them, by the number of lanes): the same counts
// with far fewer atomics on the hot bins.  Every lane of a warp runs the same iterations
// (the loop steps over warp-sized groups of pixels), as the full-warp match requires.
__global__ void __launch_bounds__(256) histogram_kernel(const float* __restrict__ it, size_t n,
                                                        double inv_max, int num_bins,
                                                        int* __restrict__ hist) {
    const int lane = threadIdx.x & 31;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t base = blockIdx.x * (size_t)blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        const size_t q = base + lane;
        int bin = -1;
        if (q < n) {
            const float s = it[q];
            if (s >= 0.0f) {
                const double pos = ((double)s * inv_max) * (double)(num_bins - 1);
                bin = (int)pos;
                if (bin >= num_bins) bin = num_bins - 1;
                else if (bin < 0) bin = 0;
            }
        }
        const unsigned peers = __match_any_sync(0xffffffffu, bin);
        if (bin >= 0 && lane == __ffs(peers) - 1) atomicAdd(hist + bin, __popc(peers));
    }
}

// One block of 1024 threads: inclusive prefix sum of the histogram in exact
// integer arithmetic, then cdf[b] = float32(prefix[b] / total) as the
// float64 scan of math_core/cuda_kernels.py:1929-1996 produces it.  Serves bin
// counts above kChunkMaxBins (cdf_chunk_kernel below serves the rest).
constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads) cdf_kernel(const int* __restrict__ hist,
                                                           int num_bins, float* __restrict__ cdf) {
    __shared__ long long warp_sums[kScanThreads / 32];
    __shared__ long long total_s;
    const int t = threadIdx.x;
    const int chunk = (num_bins + kScanThreads - 1) / kScanThreads;
    const int b0 = t * chunk;
    const int b1 = min(b0 + chunk, num_bins);
    long long local = 0;
    for (int q = b0; q < b1; ++q) local += hist[q];

    // Block-wide exclusive scan of the per-thread sums.
    const int lane = t & 31, warp = t >> 5;
    long long v = local;
    for (int o = 1; o < 32; o <<= 1) {
        const long long u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) warp_sums[warp] = v;
    __syncthreads();
    if (warp == 0) {
        long long w = warp_sums[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const long long u = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += u;
        }
        warp_sums[lane] = w;
        if (lane == 31) total_s = w;
    }
    __syncthreads();
    long long run = (v - local) + (warp > 0 ? warp_sums[warp - 1] : 0LL);
    const double total = (double)total_s;
    for (int q = b0; q < b1; ++q) {
        run += hist[q];
        cdf[q] = total > 0.0 ? (float)((double)run / total)
                             : (float)((double)q / (double)(num_bins - 1));
    }
}

// Chunked form for up to kChunkMaxBins bins (the reference's 65536): block b scans bins
// [4096 b, 4096 (b + 1)).  Every block first reads all counts, coalesced, for the sum of
// the bins before its chunk and the total (256 KiB from L2 at 65536 bins), so no block
// waits on another; then each thread takes 16 consecutive bins, the thread sums are
// scanned across the block, and each bin gets cdf = float32(float64(prefix) / total) with
// the same exact integer prefix and division as cdf_kernel.
constexpr int kChunkBins = 4096;
constexpr int kChunkThreads = 256;
constexpr int kChunkPerThread = kChunkBins / kChunkThreads;  // 16
constexpr int kChunkMaxBins = 65536;

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(kChunkThreads) cdf_chunk_kernel(const int* __restrict__ hist,
                                                                  int num_bins, float* __restrict__ cdf) {
    __shared__ long long red_before[kChunkThreads / 32], red_total[kChunkThreads / 32];
    __shared__ long long scan_s[kChunkThreads / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int start = blockIdx.x * kChunkBins;
    long long before = 0, total = 0;
    if ((num_bins & 3) == 0 && (reinterpret_cast<uintptr_t>(hist) & 15u) == 0) {
        const int4* h4 = reinterpret_cast<const int4*>(hist);
        const int n4 = num_bins >> 2, s4 = start >> 2;
#pragma unroll 4
        for (int q = t; q < n4; q += kChunkThreads) {
            const int4 v = __ldg(h4 + q);
            const long long s = (long long)v.x + v.y + v.z + v.w;
            total += s;
            if (q < s4) before += s;
        }
    } else {
#pragma unroll 4
        for (int q = t; q < num_bins; q += kChunkThreads) {
            const long long v = __ldg(hist + q);
            total += v;
            if (q < start) before += v;
        }
    }
    before = warp_sum_ll(before);
    total = warp_sum_ll(total);
    if (lane == 0) {
        red_before[warp] = before;
        red_total[warp] = total;
    }
    __syncthreads();
    before = total = 0;
#pragma unroll
    for (int w = 0; w < kChunkThreads / 32; ++w) {
        before += red_before[w];
        total += red_total[w];
    }
    // this thread's 16 bins and their sum
    const int b0 = start + t * kChunkPerThread;
    long long c[kChunkPerThread];
    long long mine = 0;
#pragma unroll
    for (int q = 0; q < kChunkPerThread; ++q) {
        c[q] = (b0 + q < num_bins) ? (long long)__ldg(hist + b0 + q) : 0LL;
        mine += c[q];
    }
    // exclusive scan of the thread sums across the block
    long long v = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) scan_s[warp] = v;
    __syncthreads();
    long long run = before + (v - mine);
    for (int w = 0; w < warp; ++w) run += scan_s[w];
    const double tot = (double)total;
#pragma unroll
    for (int q = 0; q < kChunkPerThread; ++q) {
        const int b = b0 + q;
        if (b >= num_bins) break;
        run += c[q];
        cdf[b] = tot > 0.0 ? (float)((double)run / tot) : (float)((double)b / (double)(num_bins - 1));
    }
}

// The aligned form (num_bins a multiple of 4 up to kChunkMaxBins, hist and cdf 16-byte
// aligned): blocks of 1024 threads, 4096 bins each.  Every thread reads its share of all
// counts as at most 16 independent int4 loads (one round of memory latency, where the
// form above walks 64 loads a thread) for the total and the sum before the block's
// chunk, then one int4 of the chunk itself (4 consecutive bins, coalesced); the thread
// sums are scanned across the block and each thread writes its 4 cdf values as one
// float4.  The same exact integer prefix and float64 division as cdf_kernel.
constexpr int kChunk4Threads = 1024;

__global__ void __launch_bounds__(kChunk4Threads) cdf_chunk4_kernel(const int4* __restrict__ h4, int n4,
                                                                    int num_bins, float4* __restrict__ cdf4) {
    __shared__ long long red_before[kChunk4Threads / 32], red_total[kChunk4Threads / 32];
    __shared__ long long scan_s[kChunk4Threads / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int s4 = blockIdx.x * kChunk4Threads;  // the chunk's first int4
    long long before = 0, total = 0;
#pragma unroll
    for (int r = 0; r < kChunkMaxBins / 4 / kChunk4Threads; ++r) {
        const int q = t + r * kChunk4Threads;
        if (q < n4) {
            const int4 v = __ldg(h4 + q);
            const long long s = (long long)v.x + v.y + v.z + v.w;
            total += s;
            if (q < s4) before += s;
        }
    }
    before = warp_sum_ll(before);
    total = warp_sum_ll(total);
    if (lane == 0) {
        red_before[warp] = before;
        red_total[warp] = total;
    }
    const int q = s4 + t;
    const int4 c = q < n4 ? __ldg(h4 + q) : make_int4(0, 0, 0, 0);
    const long long mine = (long long)c.x + c.y + c.z + c.w;
    long long v = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) scan_s[warp] = v;
    __syncthreads();
    before = total = 0;
    long long run = v - mine;
#pragma unroll 8
    for (int w = 0; w < kChunk4Threads / 32; ++w) {
        before += red_before[w];
        total += red_total[w];
        if (w < warp) run += scan_s[w];
    }
    if (q >= n4) return;
    run += before;
    const double tot = (double)total;
    const int b = 4 * q;
    auto value = [&](long long prefix, int bin) {
        return tot > 0.0 ? (float)((double)prefix / tot) : (float)((double)bin / (double)(num_bins - 1));
    };
    float4 out;
    run += c.x;
    out.x = value(run, b);
    run += c.y;
    out.y = value(run, b + 1);
    run += c.z;
    out.z = value(run, b + 2);
    run += c.w;
    out.w = value(run, b + 3);
    cdf4[q] = out;
}

// The CDF of a histogram: the aligned chunked form, the chunked form, or one block.
static int launch_cdf(const int32_t* hist, int num_bins, float* cdf, cudaStream_t st) {
    if (num_bins <= kChunkMaxBins && (num_bins & 3) == 0 && (reinterpret_cast<uintptr_t>(hist) & 15u) == 0 &&
        (reinterpret_cast<uintptr_t>(cdf) & 15u) == 0) {
        const int n4 = num_bins >> 2;
        cdf_chunk4_kernel<<<(n4 + kChunk4Threads - 1) / kChunk4Threads, kChunk4Threads, 0, st>>>(
            reinterpret_cast<const int4*>(hist), n4, num_bins, reinterpret_cast<float4*>(cdf));
        return check_launch("cdf_chunk4_kernel");
    }
    if (num_bins <= kChunkMaxBins) {
        const int blocks = (num_bins + kChunkBins - 1) / kChunkBins;
        cdf_chunk_kernel<<<blocks, kChunkThreads, 0, st>>>(hist, num_bins, cdf);
        return check_launch("cdf_chunk_kernel");
    }
    cdf_kernel<<<1, kScanThreads, 0, st>>>(hist, num_bins, cdf);
    return check_launch("cdf_kernel");
}

// ----------------------------------------------------------------- colour
// apply_histogram_equalization_kernel (math_core/cuda_kernels.py:2016) and
// recolor_iter_map_cuda_kernel (math_core/cuda_kernels.py:3201).
__global__ void __launch_bounds__(256) colour_kernel(const ApFrameParams p, const ApFrameBuffers b,
                                                     int hist) {
    const int i = blockIdx.x * 16 + (threadIdx.x & 15);
    const int j = blockIdx.y * 16 + (threadIdx.x >> 4);
    if (i >= p.width || j >= p.height) return;
    const size_t idx = (size_t)j * p.width + i;
    if (p.rebase_pass > 0 && b.glitch_in != nullptr && b.glitch_in[idx] == 0) return;
    const double s = (double)b.iter_map[idx];
    double r = 0.0, g = 0.0, bb = 0.0;
    if (s >= 0.0) colour_of(p, b.lut, b.cdf, hist != 0, s, r, g, bb);
    store_rgb(b.rgb, p.is_hdr, idx, r, g, bb);
}

// ---------------------------------------------------------- listed pixels
// Values computed elsewhere for a list of pixels (the Strict Metric
// re-evaluation, math_core/engine.py:191-267): iter_map = float32(value), the
// colour of the float64 value (black for value < 0 or >= max_iter), glitch
// flag cleared.
__global__ void __launch_bounds__(256) set_pixels_kernel(const ApFrameParams p, const ApFrameBuffers b,
                                                         const int32_t* __restrict__ coords,
                                                         const double* __restrict__ values, int n,
                                                         int hist) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int r = coords[2 * q], c = coords[2 * q + 1];
    if (r < 0 || r >= p.height || c < 0 || c >= p.width) return;
    const size_t idx = (size_t)r * p.width + c;
    const double s = values[q];
    b.iter_map[idx] = (float)s;
    double cr = 0.0, cg = 0.0, cb = 0.0;
    if (s >= 0.0 && s < (double)p.max_iter) colour_of(p, b.lut, b.cdf, hist != 0, s, cr, cg, cb);
    store_rgb(b.rgb, p.is_hdr, idx, cr, cg, cb);
    if (b.glitch_out) b.glitch_out[idx] = 0;
}

// ----------------------------------------------------------- rebase bins
// Glitched pixels per cell of the 16 x 16 grid the rebase loop picks its next
// reference from (math_core/engine.py:1923-1935: row bin (16 j) / H, column bin
// (16 i) / W).  One block per 256 x 16 pixel slab; shared-memory counts, then
// one atomic per non-empty cell.
__global__ void __launch_bounds__(256) glitch_bins_kernel(const uint8_t* __restrict__ g, int W, int H,
                                                          int* __restrict__ counts) {
    __shared__ int c[256];
    c[threadIdx.x] = 0;
    __syncthreads();
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i < W) {
        const int bc = min(15, (i * 16) / W);
        const int j0 = blockIdx.y * 16, j1 = min(H, j0 + 16);
        for (int j = j0; j < j1; ++j) {
            if (g[(size_t)j * W + i]) atomicAdd(&c[min(15, (j * 16) / H) * 16 + bc], 1);
        }
    }
    __syncthreads();
    if (c[threadIdx.x]) atomicAdd(counts + threadIdx.x, c[threadIdx.x]);
}

}  // namespace ap

extern "C" int ap_edge_detect(const float* iter_map, uint8_t* edge_mask, int32_t width,
                              int32_t height, float threshold, void* stream) {
    if (!iter_map || !edge_mask || width <= 0 || height <= 0) {
        ap::set_error("ap_edge_detect: bad arguments");
        return AP_E_INVALID;
    }
    dim3 grid((width + 15) / 16, (height + 15) / 16);
    ap::edge_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(iter_map, edge_mask, width,
                                                                        height, threshold);
    return ap::check_launch("edge_kernel");
}

extern "C" int ap_histogram_cdf(const float* iter_map, int32_t width, int32_t height,
                                int32_t max_iter, int32_t num_bins, int32_t* hist, float* cdf,
                                void* stream) {
    if (!iter_map || !hist || !cdf || width <= 0 || height <= 0 || num_bins < 2 ||
        num_bins > (1 << 24)) {
        ap::set_error("ap_histogram_cdf: bad arguments");
        return AP_E_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(int32_t) * (size_t)num_bins, st);
    if (e != cudaSuccess) {
        ap::set_error("ap_histogram_cdf: memset: %s", cudaGetErrorString(e));
        return AP_E_CUDA;
    }
    const size_t n = (size_t)width * height;
    const double inv_max = 1.0 / fmax(1.0, (double)max_iter);
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    ap::histogram_kernel<<<blocks, 256, 0, st>>>(iter_map, n, inv_max, num_bins, hist);
    int rc = ap::check_launch("histogram_kernel");
    if (rc != AP_OK) return rc;
    return ap::launch_cdf(hist, num_bins, cdf, st);
}

extern "C" int ap_histogram(const float* iter_map, int32_t width, int32_t height, int32_t max_iter,
                            int32_t num_bins, int32_t* hist, void* stream) {
    if (!iter_map || !hist || width < 0 || height < 0 || num_bins < 2 || num_bins > (1 << 24)) {
        ap::set_error("ap_histogram: bad arguments");
        return AP_E_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(hist, 0, sizeof(int32_t) * (size_t)num_bins, st);
    if (e != cudaSuccess) {
        ap::set_error("ap_histogram: memset: %s", cudaGetErrorString(e));
        return AP_E_CUDA;
    }
    const size_t n = (size_t)width * height;
    if (n == 0) return AP_OK;
    const double inv_max = 1.0 / fmax(1.0, (double)max_iter);
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 16) blocks = 148 * 16;
    ap::histogram_kernel<<<blocks, 256, 0, st>>>(iter_map, n, inv_max, num_bins, hist);
    return ap::check_launch("histogram_kernel");
}

extern "C" int ap_cdf_from_histogram(const int32_t* hist, int32_t num_bins, float* cdf, void* stream) {
    if (!hist || !cdf || num_bins < 2 || num_bins > (1 << 24)) {
        ap::set_error("ap_cdf_from_histogram: bad arguments");
        return AP_E_INVALID;
    }
    return ap::launch_cdf(hist, num_bins, cdf, static_cast<cudaStream_t>(stream));
}

extern "C" int ap_colour(const ApFrameParams* p, const ApFrameBuffers* b, void* stream) {
    if (!p || !b || !b->iter_map || !b->rgb || !b->lut || p->width <= 0 || p->height <= 0) {
        ap::set_error("ap_colour: bad arguments");
        return AP_E_INVALID;
    }
    const int hist = (p->scheme_id == 11 && b->cdf != nullptr) ? 1 : 0;
    if (hist && p->num_bins < 2) {
        ap::set_error("ap_colour: num_bins must be >= 2");
        return AP_E_INVALID;
    }
    dim3 grid((p->width + 15) / 16, (p->height + 15) / 16);
    ap::colour_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(*p, *b, hist);
    return ap::check_launch("colour_kernel");
}

extern "C" int ap_glitch_bins(const uint8_t* glitch_map, int32_t width, int32_t height,
                              int32_t* counts, void* stream) {
    if (!glitch_map || !counts || width <= 0 || height <= 0 || width > (1 << 26) / 16 ||
        height > (1 << 26) / 16) {
        ap::set_error("ap_glitch_bins: bad arguments");
        return AP_E_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(counts, 0, 256 * sizeof(int32_t), st);
    if (e != cudaSuccess) {
        ap::set_error("ap_glitch_bins: memset: %s", cudaGetErrorString(e));
        return AP_E_CUDA;
    }
    dim3 grid((width + 255) / 256, (height + 15) / 16);
    ap::glitch_bins_kernel<<<grid, 256, 0, st>>>(glitch_map, width, height, counts);
    return ap::check_launch("glitch_bins_kernel");
}

extern "C" int ap_set_pixels(const ApFrameParams* p, const ApFrameBuffers* b, const int32_t* coords,
                             const double* values, int32_t n, void* stream) {
    if (!p || !b || !b->iter_map || !b->rgb || !b->lut || n < 0 || (n > 0 && (!coords || !values)) ||
        p->width <= 0 || p->height <= 0) {
        ap::set_error("ap_set_pixels: bad arguments");
        return AP_E_INVALID;
    }
    if (n == 0) return AP_OK;
    const int hist = (p->scheme_id == 11 && b->cdf != nullptr) ? 1 : 0;
    ap::set_pixels_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        *p, *b, coords, values, n, hist);
    return ap::check_launch("set_pixels_kernel");
}
