// ap_batch.cu -- many tiles of uneven size, formula and max_iter in one
// persistent kernel.
//
// A tile is one coarse perturbation pass (AP_TIER_PERTURB with packed orbit and
// BLA rows, or AP_TIER_FLOATEXP32 with the FP32 form's packed inputs; no in-kernel
// colour) with its own parameters and outputs, in the single-reference form or in
// one-pass rebasing (AP_FLAG_REBASE).  Each
// tile is cut into patches of patch_w x patch_h = 256 pixels; patches are
// numbered tile after tile (the host orders tiles by estimated cost, largest
// first).  The grid holds blocks_per_sm blocks per SM for the whole batch; the
// queue is one global pixel counter.
//
// A block works in rounds.  In a round each thread runs one pixel for `quantum`
// loop steps, resumable (the per-frame kernel's pixel_begin / pixel_advance /
// rebase_advance / pixel_finish, and fe32_begin / fe32_advance / fe32_finish for FP32
// tiles, so values are identical).  A pixel that finishes is
// written out; one that does not leaves its state in the block's shared slots.  At
// the end of the round the block compacts the unfinished pixels into its first
// slots, keeping their order, so they run together in as few warps as possible in
// the next round, and the slots left over take the next pixels of the queue, all
// of them with one atomicAdd: those are consecutive pixels of a patch, neighbours
// that start together, share orbit records and branch alike.  Nothing waits on
// anything outside the block: a block whose slots are empty once the queue has run
// out exits.
#include "ap_coarse.cuh"
#include "ap_fe32.cuh"

namespace ap {

static_assert(sizeof(ApTileDesc) % 16 == 0, "tile descriptors are 16-byte aligned records");

// Threads (pixel slots) per block.  A larger block packs its unfinished pixels into
// fuller warps at each compaction: 512 slots took config 4 from 230 to 214 ms against
// 256 (with a 256-step quantum), 128 slots to 250 ms.
#ifndef AP_BATCH_THREADS
#define AP_BATCH_THREADS 512
#endif
constexpr int kBatchThreads = AP_BATCH_THREADS;

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

// The unfinished pixels of a block between rounds, one slot per thread, as a
// structure of arrays (thread q touches word q of each array: no bank conflicts).
// A stage-2 pixel keeps z itself where a stage-1 pixel keeps its delta; a one-pass
// pixel keeps its reference index m where a single-reference pixel keeps the step
// at which it entered stage 2.  The finished sample is not kept: a pixel that has
// not finished holds the interior sample.  64 bytes a slot (32 KiB for 512 slots).
struct BatchSlots {
    double zx[kBatchThreads], zy[kBatchThreads];
    double dcx[kBatchThreads], dcy[kBatchThreads];
    int idx[kBatchThreads], k[kBatchThreads], k0[kBatchThreads], k2m[kBatchThreads];
    int leaps[kBatchThreads], skipped[kBatchThreads], rebases[kBatchThreads];
    int tag[kBatchThreads];  // tile << 3 | stage << 1 | glitch
};

__device__ __forceinline__ void slot_store(BatchSlots& S, int q, const PixelRun& s, int tile, bool rebase) {
    const bool st2 = s.stage == 2;
    S.zx[q] = st2 ? s.zx : s.dzx;
    S.zy[q] = st2 ? s.zy : s.dzy;
    S.dcx[q] = s.dcx;
    S.dcy[q] = s.dcy;
    S.idx[q] = s.idx;
    S.k[q] = s.k;
    S.k0[q] = s.k0;
    S.k2m[q] = rebase ? s.m : s.k2;
    S.leaps[q] = s.leaps;
    S.skipped[q] = s.skipped;
    S.rebases[q] = s.rebases;
    S.tag[q] = (tile << 3) | (s.stage << 1) | (s.glitch ? 1 : 0);
}

// What a round reads: everything but the pixel index and its first step, which only
// the final write-out needs (fewer values live across the loop).
__device__ __forceinline__ void slot_load_run(const BatchSlots& S, int q, PixelRun& s, bool rebase) {
    const int tag = S.tag[q];
    s.stage = (tag >> 1) & 3;
    s.glitch = tag & 1;
    const double a = S.zx[q], c = S.zy[q];
    s.dzx = s.stage == 2 ? 0.0 : a;
    s.dzy = s.stage == 2 ? 0.0 : c;
    s.zx = s.stage == 2 ? a : 0.0;
    s.zy = s.stage == 2 ? c : 0.0;
    s.dcx = S.dcx[q];
    s.dcy = S.dcy[q];
    s.idx = 0;
    s.k = S.k[q];
    s.k0 = 0;
    s.m = rebase ? S.k2m[q] : s.k;
    s.k2 = rebase ? -1 : S.k2m[q];
    s.leaps = S.leaps[q];
    s.skipped = S.skipped[q];
    s.rebases = S.rebases[q];
    s.o = interior_sample();
}

// What a round changes (the tile, the offset dc, the index and the first step stay).
__device__ __forceinline__ void slot_store_run(BatchSlots& S, int q, const PixelRun& s, bool rebase) {
    const bool st2 = s.stage == 2;
    S.zx[q] = st2 ? s.zx : s.dzx;
    S.zy[q] = st2 ? s.zy : s.dzy;
    S.k[q] = s.k;
    S.k2m[q] = rebase ? s.m : s.k2;
    S.leaps[q] = s.leaps;
    S.skipped[q] = s.skipped;
    S.rebases[q] = s.rebases;
    S.tag[q] = (S.tag[q] & ~7) | (s.stage << 1) | (s.glitch ? 1 : 0);
}

// One round of the pixel in slot q (of tile t): loop steps up to the quantum; the
// pixel is written out when it finishes.  Returns true when it has not finished; its
// state is then back in slot q.  One variant per (profile, formula class, BLA,
// rebasing): separate functions, so each keeps the register allocation it has in the
// per-frame kernel.
template <int ARITH, int FT, bool BLA, bool REBASE>
__device__ __noinline__ bool slot_run(const ApTileDesc* __restrict__ t, BatchSlots& S, int q, int quantum) {
    const ApFrameBuffers b = tile_buffers(t);
    PixelRun s;
    slot_load_run(S, q, s, REBASE);
    if (REBASE)
        rebase_advance<ARITH, FT, BLA, true>(t->p, b, s, quantum);
    else
        pixel_advance<ARITH, FT, BLA, true>(t->p, b, s, quantum);
    if (s.stage == 3) {
        s.idx = S.idx[q];
        s.k0 = S.k0[q];
        pixel_finish(t->p, b, s);
        return false;
    }
    slot_store_run(S, q, s, REBASE);
    return true;
}

// FP32 tiles (AP_TIER_FLOATEXP32) keep their pixels in the same slots: the delta's
// mantissa pair (exactly, as doubles) where an FP64 pixel keeps its delta, z in stage 2
// as there, the offset dc in units of 2^-E, and the delta's exponent where an FP64
// pixel keeps its first step (an FP32 pixel takes no series start: it starts at 0).
__device__ __forceinline__ void fe32_slot_store(BatchSlots& S, int q, const Fe32Run& s, int tile, bool rebase) {
    const bool st2 = s.stage == 2;
    S.zx[q] = st2 ? s.zx : (double)s.wx;
    S.zy[q] = st2 ? s.zy : (double)s.wy;
    S.dcx[q] = s.dcx;
    S.dcy[q] = s.dcy;
    S.idx[q] = s.idx;
    S.k[q] = s.k;
    S.k0[q] = s.e;
    S.k2m[q] = rebase ? s.m : s.k2;
    S.leaps[q] = s.leaps;
    S.skipped[q] = s.skipped;
    S.rebases[q] = s.rebases;
    S.tag[q] = (tile << 3) | (s.stage << 1) | (s.glitch ? 1 : 0);
}

__device__ __forceinline__ void fe32_slot_load(const BatchSlots& S, int q, Fe32Run& s, bool rebase) {
    const int tag = S.tag[q];
    s.stage = (tag >> 1) & 3;
    s.glitch = tag & 1;
    const double a = S.zx[q], c = S.zy[q];
    const bool st2 = s.stage == 2;
    s.wx = st2 ? 0.0f : (float)a;
    s.wy = st2 ? 0.0f : (float)c;
    s.zx = st2 ? a : 0.0;
    s.zy = st2 ? c : 0.0;
    s.dcx = S.dcx[q];
    s.dcy = S.dcy[q];
    s.idx = 0;
    s.k = S.k[q];
    s.e = S.k0[q];
    s.m = rebase ? S.k2m[q] : 0;
    s.k2 = rebase ? -1 : S.k2m[q];
    s.leaps = S.leaps[q];
    s.skipped = S.skipped[q];
    s.rebases = S.rebases[q];
    s.o = interior_sample();
}

// What a round of an FP32 pixel changes (the tile, dc and the index stay).
__device__ __forceinline__ void fe32_slot_store_run(BatchSlots& S, int q, const Fe32Run& s, bool rebase) {
    const bool st2 = s.stage == 2;
    S.zx[q] = st2 ? s.zx : (double)s.wx;
    S.zy[q] = st2 ? s.zy : (double)s.wy;
    S.k[q] = s.k;
    S.k0[q] = s.e;
    S.k2m[q] = rebase ? s.m : s.k2;
    S.leaps[q] = s.leaps;
    S.skipped[q] = s.skipped;
    S.rebases[q] = s.rebases;
    S.tag[q] = (S.tag[q] & ~7) | (s.stage << 1) | (s.glitch ? 1 : 0);
}

// One round of an FP32 pixel (as slot_run).
template <int FT, bool BLA, bool REBASE>
__device__ __noinline__ bool fe32_slot_run(const ApTileDesc* __restrict__ t, BatchSlots& S, int q, int quantum) {
    const ApFrameBuffers b = tile_buffers(t);
    Fe32Run s;
    fe32_slot_load(S, q, s, REBASE);
    fe32_advance<FT, BLA, REBASE, true>(t->p, b, s, quantum);
    if (s.stage == 3) {
        s.idx = S.idx[q];
        fe32_finish(t->p, b, s);
        return false;
    }
    fe32_slot_store_run(S, q, s, REBASE);
    return true;
}

// FP32 formula dispatch (Burning Ship types take no leaps, as in the per-frame pass).
__device__ __forceinline__ bool fe32_batch_run(const ApTileDesc* t, BatchSlots& S, int q, int quantum) {
    const bool bla = t->p.bla_levels > 1 && t->bla_packed != nullptr;
    const bool rebase = (t->p.flags & AP_FLAG_REBASE) != 0;
    switch (t->p.fractal_type) {
    case 1:
    case 3:
        return rebase ? fe32_slot_run<kFtShip, false, true>(t, S, q, quantum)
                      : fe32_slot_run<kFtShip, false, false>(t, S, q, quantum);
    case 4:
        if (rebase)
            return bla ? fe32_slot_run<kFtMulti, true, true>(t, S, q, quantum)
                       : fe32_slot_run<kFtMulti, false, true>(t, S, q, quantum);
        return bla ? fe32_slot_run<kFtMulti, true, false>(t, S, q, quantum)
                   : fe32_slot_run<kFtMulti, false, false>(t, S, q, quantum);
    default:
        if (rebase)
            return bla ? fe32_slot_run<kFtQuad, true, true>(t, S, q, quantum)
                       : fe32_slot_run<kFtQuad, false, true>(t, S, q, quantum);
        return bla ? fe32_slot_run<kFtQuad, true, false>(t, S, q, quantum)
                   : fe32_slot_run<kFtQuad, false, false>(t, S, q, quantum);
    }
}

// Formula dispatch.  AP_ARITH_FAST serves one-pass tiles only; a FAST batch's
// single-reference tiles (Julia types) run the CUDA-source profile.
template <int ARITH>
__device__ __forceinline__ bool batch_run(const ApTileDesc* t, BatchSlots& S, int q, int quantum) {
    constexpr int kPlain = (ARITH == AP_ARITH_FAST) ? AP_ARITH_REF_CUDA : ARITH;
    if (t->p.tier == AP_TIER_FLOATEXP32) return fe32_batch_run(t, S, q, quantum);
    const bool bla = t->p.bla_levels > 1 && t->bla_packed != nullptr;
    if (t->p.flags & AP_FLAG_REBASE) {
        switch (t->p.fractal_type) {
        case 1: return slot_run<ARITH, kFtShip, false, true>(t, S, q, quantum);
        case 4:
            return bla ? slot_run<ARITH, kFtMulti, true, true>(t, S, q, quantum)
                       : slot_run<ARITH, kFtMulti, false, true>(t, S, q, quantum);
        default:
            return bla ? slot_run<ARITH, kFtQuad, true, true>(t, S, q, quantum)
                       : slot_run<ARITH, kFtQuad, false, true>(t, S, q, quantum);
        }
    }
    switch (t->p.fractal_type) {
    case 1:
    case 3: return slot_run<kPlain, kFtShip, false, false>(t, S, q, quantum);
    case 4:
        return bla ? slot_run<kPlain, kFtMulti, true, false>(t, S, q, quantum)
                   : slot_run<kPlain, kFtMulti, false, false>(t, S, q, quantum);
    default:
        return bla ? slot_run<kPlain, kFtQuad, true, false>(t, S, q, quantum)
                   : slot_run<kPlain, kFtQuad, false, false>(t, S, q, quantum);
    }
}

// A fresh pixel (i, j) of tile t into slot q (pixel_begin); false when it has no work.
// The set-up differs between formulas only in the series start, which Burning Ship
// types do not take.
template <int ARITH>
__device__ __noinline__ bool slot_begin(const ApTileDesc* __restrict__ t, int tile, BatchSlots& S, int q, int i,
                                        int j) {
    const bool rebase = (t->p.flags & AP_FLAG_REBASE) != 0;
    if (t->p.tier == AP_TIER_FLOATEXP32) {
        Fe32Run f;
        const bool ok = fe32_begin(t->p, tile_buffers(t), i, j, f);
        if (ok) fe32_slot_store(S, q, f, tile, rebase);
        return ok;
    }
    PixelRun s;
    const bool ship = t->p.fractal_type == 1 || t->p.fractal_type == 3;
    const bool ok = ship ? pixel_begin<ARITH, kFtShip>(t->p, tile_buffers(t), i, j, s)
                         : pixel_begin<ARITH, kFtQuad>(t->p, tile_buffers(t), i, j, s);
    if (ok) slot_store(S, q, s, tile, rebase);
    return ok;
}

// Pixel u of the batch (patches of 256 pixels, numbered tile after tile; row-major in a
// patch) -> its tile and its (i, j); false when it falls outside the tile.
__device__ __forceinline__ bool batch_pixel_at(const ApTileDesc* __restrict__ tiles,
                                               const int64_t* __restrict__ first, int n, int patch_w,
                                               int patch_h, long long u, int* tile, int* i, int* j) {
    const long long item = u >> 8;  // the patch
    const int q = (int)(u & 255);
    int lo = 0, hi = n - 1;  // last tile whose first patch <= item
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (first[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    *tile = lo;
    const ApTileDesc* t = tiles + lo;
    const long long local = item - first[lo];
    const int px = (t->p.width + patch_w - 1) / patch_w;
    *i = (int)(local % px) * patch_w + q % patch_w;
    *j = (int)(local / px) * patch_h + q / patch_w;
    return *i < t->p.width && *j < t->p.height;
}

template <int ARITH, int MINB>
__global__ void __launch_bounds__(kBatchThreads, MINB * 256 / kBatchThreads) batch_kernel(const ApTileDesc* __restrict__ tiles,
                                                                    const int64_t* __restrict__ first,
                                                                    int n, int patch_w, int patch_h,
                                                                    int quantum,
                                                                    unsigned long long* head) {
    __shared__ BatchSlots S;
    __shared__ int warp_live[kBatchThreads / 32];
    __shared__ int live_s, drained_s;
    __shared__ unsigned long long base_s;
    const unsigned full = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long total = first[n] * 256;
    if (tid == 0) {
        live_s = 0;
        drained_s = 0;
    }
    __syncthreads();
    for (;;) {
        // the slots past the live pixels take the next pixels of the queue
        const int live = live_s;
        const bool take = !drained_s && live < kBatchThreads;
        if (tid == 0 && take) base_s = atomicAdd(head, (unsigned long long)(kBatchThreads - live));
        __syncthreads();
        bool running = false;
        int tile = 0;
        if (tid < live) {
            tile = S.tag[tid] >> 3;
            running = true;
        } else if (take) {
            const long long u = (long long)base_s + (tid - live);
            int i = 0, j = 0;
            if (u < total && batch_pixel_at(tiles, first, n, patch_w, patch_h, u, &tile, &i, &j))
                running = slot_begin<ARITH>(tiles + tile, tile, S, tid, i, j);
        }
        if (running) running = batch_run<ARITH>(tiles + tile, S, tid, quantum);
        // compact the unfinished pixels into the first slots, in order
        const unsigned bal = __ballot_sync(full, running);
        if (lane == 0) warp_live[warp] = __popc(bal);
        __syncthreads();
        int pos = __popc(bal & ((1u << lane) - 1u)), now = 0;
#pragma unroll
        for (int w = 0; w < kBatchThreads / 32; ++w) {
            pos += (w < warp) ? warp_live[w] : 0;
            now += warp_live[w];
        }
        double zx = 0.0, zy = 0.0, dcx = 0.0, dcy = 0.0;
        int w0 = 0, w1 = 0, w2 = 0, w3 = 0, w4 = 0, w5 = 0, w6 = 0, w7 = 0;
        if (running) {
            zx = S.zx[tid], zy = S.zy[tid], dcx = S.dcx[tid], dcy = S.dcy[tid];
            w0 = S.idx[tid], w1 = S.k[tid], w2 = S.k0[tid], w3 = S.k2m[tid];
            w4 = S.leaps[tid], w5 = S.skipped[tid], w6 = S.rebases[tid], w7 = S.tag[tid];
        }
        __syncthreads();
        if (running && pos != tid) {
            S.zx[pos] = zx, S.zy[pos] = zy, S.dcx[pos] = dcx, S.dcy[pos] = dcy;
            S.idx[pos] = w0, S.k[pos] = w1, S.k0[pos] = w2, S.k2m[pos] = w3;
            S.leaps[pos] = w4, S.skipped[pos] = w5, S.rebases[pos] = w6, S.tag[pos] = w7;
        }
        if (tid == 0) {
            live_s = now;
            if (take && base_s + (unsigned long long)(kBatchThreads - live) >= (unsigned long long)total)
                drained_s = 1;
        }
        __syncthreads();
        if (drained_s && live_s == 0) break;
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
    if (!tiles || !first_patch || n < 1 || n > (1 << 26) || patch_w < 1 || patch_h < 1 ||
        patch_w * patch_h != 256) {
        ap::set_error("ap_batch_plan: bad arguments (1 <= n <= 2^26, patch_w * patch_h == 256)");
        return AP_E_INVALID;
    }
    int64_t acc = 0;
    // the batch's arithmetic profile: its FP64 tiles'; FP32 tiles have their own form
    int a0 = -1;
    for (int q = 0; q < n && a0 < 0; ++q)
        if (tiles[q].p.tier == AP_TIER_PERTURB)
            a0 = tiles[q].p.arith == AP_ARITH_FAST ? AP_ARITH_REF_CUDA : tiles[q].p.arith;
    for (int q = 0; q < n; ++q) {
        const ApTileDesc& t = tiles[q];
        const ApFrameParams& p = t.p;
        const bool fe32 = p.tier == AP_TIER_FLOATEXP32;
        if ((p.tier != AP_TIER_PERTURB && !fe32) || (fe32 && p.bbsa_skip > 0) || p.mode != AP_MODE_COARSE ||
            !(p.flags & AP_FLAG_NO_RGB) ||
            p.rebase_pass != 0 || p.width < 1 || p.height < 1 || p.factor < 1 || p.max_iter < 0 ||
            p.fractal_type < 0 || p.fractal_type > 4 || p.ref_len < 0 || p.bla_levels > 16 ||
            (p.fractal_type == 4 && (p.gen_n < 1 || p.gen_n > 64)) || !t.orbit_packed ||
            !t.iter_map || (p.bla_levels > 1 && !t.bla_packed) ||
            (t.counters && (reinterpret_cast<uintptr_t>(t.counters) & 15u)) ||
            (long long)p.width * p.height >= (1LL << 31) ||
            ((p.flags & AP_FLAG_REBASE) && (p.fractal_type == 2 || p.fractal_type == 3 || p.ref_len < 1))) {
            ap::set_error("ap_batch_plan: tile %d is not a coarse AP_TIER_PERTURB or AP_TIER_FLOATEXP32 "
                          "pass on packed inputs without in-kernel colour", q);
            return AP_E_INVALID;
        }
        // one profile per batch; AP_ARITH_FAST is one-pass rebasing's own step, and a
        // FAST batch's single-reference tiles carry the CUDA-source profile they run in
        const int aq = p.arith == AP_ARITH_FAST ? AP_ARITH_REF_CUDA : p.arith;
        if (!fe32 && (aq != a0 || (p.arith == AP_ARITH_FAST && !(p.flags & AP_FLAG_REBASE)) ||
            (p.arith != AP_ARITH_REF_CPU && p.arith != AP_ARITH_REF_CUDA && p.arith != AP_ARITH_FAST))) {
            ap::set_error("ap_batch_plan: every tile of a batch uses one arithmetic profile "
                          "(AP_ARITH_FAST for one-pass tiles only, beside AP_ARITH_REF_CUDA)");
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
                               int32_t blocks_per_sm, int32_t min_blocks, int32_t quantum,
                               unsigned long long* queue_head, void* stream) {
    if (!tiles || !first_patch || !queue_head || n < 1 || n > (1 << 26) || patch_w < 1 || patch_h < 1 ||
        patch_w * patch_h != 256 || blocks_per_sm < 1 || blocks_per_sm > 32 ||
        (min_blocks != 4 && min_blocks != 6) || quantum < 1 || quantum > (1 << 20) ||
        (arith != AP_ARITH_REF_CPU && arith != AP_ARITH_REF_CUDA && arith != AP_ARITH_FAST)) {
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
#define AP_BATCH_LAUNCH(A, M)                                                                              \
    ap::batch_kernel<A, M><<<grid, ap::kBatchThreads, 0, st>>>(tiles, first_patch, n, patch_w, patch_h, \
                                                               quantum, queue_head)
    if (arith == AP_ARITH_REF_CPU) {
        if (min_blocks == 6) AP_BATCH_LAUNCH(AP_ARITH_REF_CPU, 6);
        else AP_BATCH_LAUNCH(AP_ARITH_REF_CPU, 4);
    } else if (arith == AP_ARITH_REF_CUDA) {
        if (min_blocks == 6) AP_BATCH_LAUNCH(AP_ARITH_REF_CUDA, 6);
        else AP_BATCH_LAUNCH(AP_ARITH_REF_CUDA, 4);
    } else {
        if (min_blocks == 6) AP_BATCH_LAUNCH(AP_ARITH_FAST, 6);
        else AP_BATCH_LAUNCH(AP_ARITH_FAST, 4);
    }
#undef AP_BATCH_LAUNCH
    return ap::check_launch("batch_kernel");
}
