// ap_batch.cu -- many tiles of uneven size, formula and max_iter in one
// persistent kernel.
//
// A tile is one coarse perturbation pass (AP_TIER_PERTURB, packed orbit and
// BLA rows, no in-kernel colour) with its own parameters and outputs.  Each
// tile is cut into patches of patch_w x patch_h = 256 pixels; patches are
// numbered tile after tile (the host orders tiles by estimated cost, largest
// first).  The grid holds blocks_per_sm blocks per SM for the whole batch; each
// warp takes the next eighth of a patch (32 pixels) from one global counter
// (atomicAdd), looks its tile up by binary search over the tiles' first patch
// numbers, evaluates its pixels with coarse_pixel (the per-frame kernel's code, so
// values are identical) and takes the next, until the counter passes the end.
// Nothing waits on anything: a warp that finds the queue empty exits.
#include "ap_coarse.cuh"

namespace ap {

static_assert(sizeof(ApTileDesc) % 16 == 0, "tile descriptors are 16-byte aligned records");

// One variant of the pixel loop per (formula class, BLA): separate functions, so
// each keeps the register allocation it has in the per-frame kernel.
template <int ARITH, int FT, bool BLA>
__device__ __noinline__ void tile_pixel(const ApTileDesc* __restrict__ t, int i, int j) {
    ApFrameBuffers b{};
    b.orbit_packed = t->orbit_packed;
    b.bla_packed = t->bla_packed;
    b.iter_map = t->iter_map;
    b.kmap = t->kmap;
    b.s64 = t->s64;
    b.glitch_out = t->glitch_out;
    b.counters = t->counters;
    coarse_pixel<ARITH, FT, BLA>(t->p, b, i, j);
}

template <int ARITH>
__device__ __forceinline__ void batch_pixel(const ApTileDesc* t, int i, int j) {
    const bool bla = t->p.bla_levels > 1 && t->bla_packed != nullptr;
    switch (t->p.fractal_type) {
    case 1:
    case 3: tile_pixel<ARITH, kFtShip, false>(t, i, j); break;
    case 4:
        if (bla) tile_pixel<ARITH, kFtMulti, true>(t, i, j);
        else tile_pixel<ARITH, kFtMulti, false>(t, i, j);
        break;
    default:
        if (bla) tile_pixel<ARITH, kFtQuad, true>(t, i, j);
        else tile_pixel<ARITH, kFtQuad, false>(t, i, j);
        break;
    }
}

template <int ARITH, int MINB>
__global__ void __launch_bounds__(256, MINB) batch_kernel(const ApTileDesc* __restrict__ tiles,
                                                          const int64_t* __restrict__ first,
                                                          int n, int patch_w, int patch_h,
                                                          unsigned long long* head) {
    // Each warp takes the next eighth of a patch (32 of its 256 pixels) on its own:
    // a warp that finishes early does not wait for the slow warps of its block.
    const long long total = first[n] * 8;
    const int lane = threadIdx.x & 31;
    for (;;) {
        unsigned long long got = 0;
        if (lane == 0) got = atomicAdd(head, 1ULL);
        const long long unit = (long long)__shfl_sync(0xffffffffu, got, 0);
        if (unit >= total) break;
        const long long item = unit >> 3;  // the patch
        const int q = (int)(unit & 7) * 32 + lane;  // pixel of the patch, row-major
        const int tx = q % patch_w, ty = q / patch_w;
        int lo = 0, hi = n - 1;  // last tile whose first patch <= item
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (first[mid] <= item) lo = mid;
            else hi = mid - 1;
        }
        const ApTileDesc& t = tiles[lo];
        const long long local = item - first[lo];
        const int px = (t.p.width + patch_w - 1) / patch_w;
        const int i = (int)(local % px) * patch_w + tx;
        const int j = (int)(local / px) * patch_h + ty;
        if (i < t.p.width && j < t.p.height) batch_pixel<ARITH>(&t, i, j);
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
            (long long)p.width * p.height >= (1LL << 31)) {
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
