// ap_perturb_fast.cu -- the per-frame coarse-pass kernel over coarse_pixel
// (ap_coarse.cuh): one thread per pixel on square tiles, 8 x 4 pixels per warp.  Picked by
// ap_render_pass for AP_TIER_PERTURB coarse passes without in-kernel colour
// when the buffers carry the packed orbit and, with BLA, the packed table.
#include "ap_coarse.cuh"

namespace ap {

#ifndef AP_REBASE_MIN_BLOCKS
#define AP_REBASE_MIN_BLOCKS 4
#endif
// Tiles of kCoarseTile x kCoarseTile pixels per block (16 or 8), warps of 8 x 4 pixels.
#ifndef AP_COARSE_TILE
#define AP_COARSE_TILE 8
#endif
constexpr int kCoarseTile = AP_COARSE_TILE;
constexpr int kCoarseThreads = kCoarseTile * kCoarseTile;
constexpr int kCoarseScale = 256 / kCoarseThreads;  // blocks per 256-thread register budget

template <int ARITH, int FT, bool BLA, bool REBASE>
__global__ void __launch_bounds__(kCoarseThreads, (REBASE ? AP_REBASE_MIN_BLOCKS : 4) * kCoarseScale)
    perturb_coarse_kernel(const ApFrameParams p, const ApFrameBuffers b, int row0, int row_end) {
    // each warp takes an 8 x 4 patch of its block's pixels: neighbours follow similar
    // paths through the loop, so compact warps diverge less; rows [row0, row_end) of
    // the frame (a whole frame, or one band of a split frame)
    constexpr int kWarpsPerRow = kCoarseTile / 8;
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int i = blockIdx.x * kCoarseTile + (w % kWarpsPerRow) * 8 + (l & 7);
    const int j = row0 + blockIdx.y * kCoarseTile + (w / kWarpsPerRow) * 4 + (l >> 3);
    if (i >= p.width || j >= row_end) return;
    coarse_pixel<ARITH, FT, BLA, REBASE>(p, b, i, j);
}

template <int ARITH, int FT>
static void launch_ft(const ApFrameParams& p, const ApFrameBuffers& b, int r0, int r1, cudaStream_t st) {
    dim3 grid((p.width + kCoarseTile - 1) / kCoarseTile, (r1 - r0 + kCoarseTile - 1) / kCoarseTile);
    if (grid.y == 0) return;
    const bool rebase = (p.flags & AP_FLAG_REBASE) != 0;
    constexpr int T = kCoarseThreads;
    if constexpr (ARITH == AP_ARITH_FAST) {  // validated: AP_ARITH_FAST passes are rebasing passes
        if (p.bla_levels > 1) perturb_coarse_kernel<ARITH, FT, true, true><<<grid, T, 0, st>>>(p, b, r0, r1);
        else perturb_coarse_kernel<ARITH, FT, false, true><<<grid, T, 0, st>>>(p, b, r0, r1);
    } else if (p.bla_levels > 1) {
        if (rebase) perturb_coarse_kernel<ARITH, FT, true, true><<<grid, T, 0, st>>>(p, b, r0, r1);
        else perturb_coarse_kernel<ARITH, FT, true, false><<<grid, T, 0, st>>>(p, b, r0, r1);
    } else {
        if (rebase) perturb_coarse_kernel<ARITH, FT, false, true><<<grid, T, 0, st>>>(p, b, r0, r1);
        else perturb_coarse_kernel<ARITH, FT, false, false><<<grid, T, 0, st>>>(p, b, r0, r1);
    }
}

template <int ARITH>
static void launch_arith(const ApFrameParams& p, const ApFrameBuffers& b, int r0, int r1, cudaStream_t st) {
    switch (p.fractal_type) {
    case 1:
    case 3: launch_ft<ARITH, kFtShip>(p, b, r0, r1, st); break;
    case 4: launch_ft<ARITH, kFtMulti>(p, b, r0, r1, st); break;
    default: launch_ft<ARITH, kFtQuad>(p, b, r0, r1, st); break;
    }
}

// Rows [row0, row0 + rows) of the frame p; AP_E_UNSUPPORTED when the pass is not one
// this kernel serves.
int launch_perturb_fast_rows(const ApFrameParams& p, const ApFrameBuffers& b, int row0, int rows,
                             cudaStream_t st) {
    const bool bla = p.bla_levels > 1 && (p.fractal_type == 0 || p.fractal_type == 2 ||
                                          p.fractal_type == 4);
    if (p.tier != AP_TIER_PERTURB || p.mode != AP_MODE_COARSE || !(p.flags & AP_FLAG_NO_RGB) ||
        b.orbit_packed == nullptr || (bla && b.bla_packed == nullptr) || p.bla_levels > 16 ||
        (long long)p.width * p.height >= (1LL << 31))
        return AP_E_UNSUPPORTED;
    ApFrameParams q = p;
    if (!bla) q.bla_levels = 0;
    const int r1 = row0 + rows;
    if (q.arith == AP_ARITH_REF_CPU) launch_arith<AP_ARITH_REF_CPU>(q, b, row0, r1, st);
    else if (q.arith == AP_ARITH_FAST) launch_arith<AP_ARITH_FAST>(q, b, row0, r1, st);
    else launch_arith<AP_ARITH_REF_CUDA>(q, b, row0, r1, st);
    return check_launch("perturb_coarse_kernel");
}

int launch_perturb_fast(const ApFrameParams& p, const ApFrameBuffers& b, cudaStream_t st) {
    return launch_perturb_fast_rows(p, b, 0, p.height, st);
}

}  // namespace ap
