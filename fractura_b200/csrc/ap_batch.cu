// ap_batch.cu -- many tiles of uneven size, formula and max_iter in one
// persistent kernel.
//
// A tile is one coarse perturbation pass (AP_TIER_PERTURB, packed orbit and
// BLA rows, no in-kernel colour) with its own parameters and outputs, in the
// single-reference form or in one-pass rebasing (AP_FLAG_REBASE).  Each
// tile is cut into patches of patch_w x patch_h = 256 pixels; patches are
// numbered tile after tile (the host orders tiles by estimated cost, largest
// first).  The grid holds blocks_per_sm blocks per SM for the whole batch.  The
// queue is one global pixel counter.  Each lane of a warp holds one pixel as a
// resumable PixelRun (the per-frame kernel's pixel_begin / pixel_advance /
// pixel_finish, so values are identical) and runs it for kQuantum loop steps at a
// time.  Between quanta, once kRefill or more lanes are idle (or all are), the warp
// takes that many consecutive pixels with one atomicAdd, so the new pixels are
// neighbours that start together and share orbit records; each lane looks its
// pixel's tile up by binary search over the tiles' first patch numbers.  Nothing
// waits on anything: a warp whose lanes all find the queue empty exits.
#include "ap_coarse.cuh"

namespace ap {

static_assert(sizeof(ApTileDesc) % 16 == 0, "tile descriptors are 16-byte aligned records");

// Steps a lane runs on its pixel before the warp lets lanes whose pixel finished take
// new ones (lanes wait at most this long for each other), and the number of idle lanes
// that triggers a refill.  Refilling single lanes scatters the warp's orbit indices
// (one record load per lane instead of one per warp).  On the 64-tile batch quanta
// 96-160 with thresholds 16-20 are equally fast (within 1 %); threshold 12 and below,
// or quanta of 512 and above, are slower (quanta 96-2048, thresholds 8-32 tried).
#ifndef AP_BATCH_QUANTUM
#define AP_BATCH_QUANTUM 128
#endif
#ifndef AP_BATCH_REFILL
#define AP_BATCH_REFILL 16
#endif
constexpr int kQuantum = AP_BATCH_QUANTUM;
constexpr int kRefill = AP_BATCH_REFILL;

inline __device__ ApFrameBuffers tile_buffers(const ApTileDesc* t) {
    ApFrameBuffers b{};
    b.orbit_packed = t->orbit_packed;
    b.bla_packed = t->bla_packed;
    b.iter_map = t->iter_map;
    b.kmap = t->kmap;
    b.s64 = t->s64;
    b.glitch_out = t->glitch_out;
    b.counters = t->counters;
    return b;
}

// One variant of the pixel loop per (formula class, BLA): separate functions, so
// each keeps the register allocation it has in the per-frame kernel.
template <int ARITH, int FT, bool BLA>
__device__ __noinline__ void tile_advance(const ApTileDesc* __restrict__ t, PixelRun& s) {
    pixel_advance<ARITH, FT, BLA, true>(t->p, tile_buffers(t), s, kQuantum);
}

// The same for tiles in one-pass rebasing (AP_FLAG_REBASE; formula types 0, 1, 4).
template <int ARITH, int FT, bool BLA>
__device__ __noinline__ void tile_rebase_advance(const ApTileDesc* __restrict__ t, PixelRun& s) {
    rebase_advance<ARITH, FT, BLA, true>(t->p, tile_buffers(t), s, kQuantum);
}

template <int ARITH>
__device__ __forceinline__ void batch_advance(const ApTileDesc* t, PixelRun& s) {
    const bool bla = t->p.bla_levels > 1 && t->bla_packed != nullptr;
    if (t->p.flags & AP_FLAG_REBASE) {
        switch (t->p.fractal_type) {
        case 1: tile_rebase_advance<ARITH, kFtShip, false>(t, s); break;
        case 4:
            if (bla) tile_rebase_advance<ARITH, kFtMulti, true>(t, s);
            else tile_rebase_advance<ARITH, kFtMulti, false>(t, s);
            break;
        default:
            if (bla) tile_rebase_advance<ARITH, kFtQuad, true>(t, s);
            else tile_rebase_advance<ARITH, kFtQuad, false>(t, s);
            break;
        }
        return;
    }
    switch (t->p.fractal_type) {
    case 1:
    case 3: tile_advance<ARITH, kFtShip, false>(t, s); break;
    case 4:
        if (bla) tile_advance<ARITH, kFtMulti, true>(t, s);
        else tile_advance<ARITH, kFtMulti, false>(t, s);
        break;
    default:
        if (bla) tile_advance<ARITH, kFtQuad, true>(t, s);
        else tile_advance<ARITH, kFtQuad, false>(t, s);
        break;
    }
}

// Pixel u of the batch (patches of 256 pixels, numbered tile after tile; row-major in a
// patch) -> its tile and its (i, j); false when it falls outside the tile.
__device__ __forceinline__ bool batch_pixel_at(const ApTileDesc* __restrict__ tiles,
                                               const int64_t* __restrict__ first, int n, int patch_w,
                                               int patch_h, long long u, const ApTileDesc** t, int* i,
                                               int* j) {
    const long long item = u >> 8;  // the patch
    const int q = (int)(u & 255);
    int lo = 0, hi = n - 1;  // last tile whose first patch <= item
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (first[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    *t = tiles + lo;
    const long long local = item - first[lo];
    const int px = ((*t)->p.width + patch_w - 1) / patch_w;
    *i = (int)(local % px) * patch_w + q % patch_w;
    *j = (int)(local / px) * patch_h + q / patch_w;
    return *i < (*t)->p.width && *j < (*t)->p.height;
}

template <int ARITH, int MINB>
__global__ void __launch_bounds__(256, MINB) batch_kernel(const ApTileDesc* __restrict__ tiles,
                                                          const int64_t* __restrict__ first,
                                                          int n, int patch_w, int patch_h,
                                                          unsigned long long* head) {
    // Lane-level work stealing: a lane runs its pixel for up to kQuantum loop
    // iterations; then, if kRefill or more lanes are idle (or none is busy), the idle
    // lanes take the next pixels of the queue (one atomicAdd per warp for all of
    // them), so a warp does not idle on one long pixel while its other lanes' pixels
    // are done.
    const long long total = first[n] * 256;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    PixelRun s;
    const ApTileDesc* t = nullptr;
    bool active = false, drained = false;
    for (;;) {
        const unsigned need = __ballot_sync(full, !active && !drained);
        const unsigned busy = __ballot_sync(full, active);
        if (need && (__popc(need) >= kRefill || busy == 0)) {
            const int leader = __ffs(need) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(head, (unsigned long long)__popc(need));
            base = __shfl_sync(full, base, leader);
            if (!active && !drained) {
                const long long u = (long long)base + __popc(need & ((1u << lane) - 1u));
                int i = 0, j = 0;
                if (u >= total) {
                    drained = true;
                } else if (batch_pixel_at(tiles, first, n, patch_w, patch_h, u, &t, &i, &j)) {
                    // the set-up differs between formulas only in the series start,
                    // which Burning Ship types do not take
                    const bool ship = t->p.fractal_type == 1 || t->p.fractal_type == 3;
                    active = ship ? pixel_begin<ARITH, kFtShip>(t->p, tile_buffers(t), i, j, s)
                                  : pixel_begin<ARITH, kFtQuad>(t->p, tile_buffers(t), i, j, s);
                }
            }
        }
        if (__ballot_sync(full, active) == 0) {
            if (__all_sync(full, drained)) break;
            continue;
        }
        if (active) {
            batch_advance<ARITH>(t, s);
            if (s.stage == 3) {
                pixel_finish(t->p, tile_buffers(t), s);
                active = false;
            }
        }
    }
}

static int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    return n;
}

}  // namespace ap

extern "C" int ap_batch_plan(const ApTileDesc* tiles, int32_t n, int32_t patch_w, int32_t patch_h,
                             int64_t* first_patch) {
    if (!tiles || !first_patch || n < 1 || patch_w < 1 || patch_h < 1 || patch_w * patch_h != 256) {
        ap::set_error("ap_batch_plan: bad arguments (n >= 1, patch_w * patch_h == 256)");
        return AP_E_INVALID;
    }
    int64_t acc = 0;
    for (int q = 0; q < n; ++q) {
        const ApTileDesc& t = tiles[q];
        const ApFrameParams& p = t.p;
        if (p.tier != AP_TIER_PERTURB || p.mode != AP_MODE_COARSE || !(p.flags & AP_FLAG_NO_RGB) ||
            p.rebase_pass != 0 || p.width < 1 || p.height < 1 || p.factor < 1 || p.max_iter < 0 ||
            p.fractal_type < 0 || p.fractal_type > 4 || p.ref_len < 0 || p.bla_levels > 16 ||
            (p.fractal_type == 4 && (p.gen_n < 1 || p.gen_n > 64)) || !t.orbit_packed ||
            !t.iter_map || (p.bla_levels > 1 && !t.bla_packed) ||
            (t.counters && (reinterpret_cast<uintptr_t>(t.counters) & 15u)) ||
            (long long)p.width * p.height >= (1LL << 31) ||
            ((p.flags & AP_FLAG_REBASE) && (p.fractal_type == 2 || p.fractal_type == 3 || p.ref_len < 1))) {
            ap::set_error("ap_batch_plan: tile %d is not a coarse AP_TIER_PERTURB pass on packed "
                          "inputs without in-kernel colour", q);
            return AP_E_INVALID;
        }
        if (p.arith != tiles[0].p.arith) {
            ap::set_error("ap_batch_plan: every tile of a batch uses one arithmetic profile");
            return AP_E_INVALID;
        }
        first_patch[q] = acc;
        acc += (int64_t)((p.width + patch_w - 1) / patch_w) * ((p.height + patch_h - 1) / patch_h);
    }
    first_patch[n] = acc;
    return AP_OK;
}

extern "C" int ap_render_batch(const ApTileDesc* tiles, const int64_t* first_patch, int32_t n,
                               int32_t arith, int32_t patch_w, int32_t patch_h,
                               int32_t blocks_per_sm, int32_t min_blocks,
                               unsigned long long* queue_head, void* stream) {
    if (!tiles || !first_patch || !queue_head || n < 1 || patch_w < 1 || patch_h < 1 ||
        patch_w * patch_h != 256 || blocks_per_sm < 1 || blocks_per_sm > 32 ||
        (min_blocks != 4 && min_blocks != 6) ||
        (arith != AP_ARITH_REF_CPU && arith != AP_ARITH_REF_CUDA)) {
        ap::set_error("ap_render_batch: bad arguments");
        return AP_E_INVALID;
    }
    const int sms = ap::sm_count();
    if (sms <= 0) {
        ap::set_error("ap_render_batch: no CUDA device");
        return AP_E_CUDA;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(queue_head, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) {
        ap::set_error("ap_render_batch: memset: %s", cudaGetErrorString(e));
        return AP_E_CUDA;
    }
    const int grid = sms * blocks_per_sm;
    if (arith == AP_ARITH_REF_CPU) {
        if (min_blocks == 6)
            ap::batch_kernel<AP_ARITH_REF_CPU, 6><<<grid, 256, 0, st>>>(tiles, first_patch, n, patch_w, patch_h, queue_head);
        else
            ap::batch_kernel<AP_ARITH_REF_CPU, 4><<<grid, 256, 0, st>>>(tiles, first_patch, n, patch_w, patch_h, queue_head);
    } else {
        if (min_blocks == 6)
            ap::batch_kernel<AP_ARITH_REF_CUDA, 6><<<grid, 256, 0, st>>>(tiles, first_patch, n, patch_w, patch_h, queue_head);
        else
            ap::batch_kernel<AP_ARITH_REF_CUDA, 4><<<grid, 256, 0, st>>>(tiles, first_patch, n, patch_w, patch_h, queue_head);
    }
    return ap::check_launch("batch_kernel");
}
