// ap_fe32.cu -- FP32-mantissa FloatExp perturbation (AP_TIER_FLOATEXP32): the packing
// of its inputs (ap_pack_fe32) and the per-frame coarse pass.  The pixel's arithmetic
// is in ap_fe32.cuh, shared with the batch kernel.
#include "ap_fe32.cuh"

namespace ap {

// Split a double into (float mantissa in [1, 2), exponent); 0 -> (0, 0).
__device__ __forceinline__ void split_pair(double re, double im, float& mr, float& mi, int& e) {
    const double m = fmax(fabs(re), fabs(im));
    if (!(m > 0.0) || !isfinite(m)) {
        mr = mi = 0.0f;
        e = 0;
        return;
    }
    int ex = ((int)((__double_as_longlong(m) >> 52) & 0x7ff)) - 1023;
    if (ex < -1022) ex = ilogb(m);  // subnormal
    const double s = ldexp(1.0, -ex);
    mr = (float)(re * s);
    mi = (float)(im * s);
    e = ex;
}

__global__ void __launch_bounds__(256) pack_fe32_kernel(const double4* __restrict__ orb, int n,
                                                        const double* __restrict__ T, int levels,
                                                        int ref_len, float4* __restrict__ orb32,
                                                        double* __restrict__ Rs,
                                                        Fe32Bla* __restrict__ AB) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) {
        const double4 Z = orb[t];
        // .w = 1 marks a close approach (|Z|^2 < 2^-100) that takes the FP64 slow path
        const double r2 = Z.x * Z.x + Z.y * Z.y;
        orb32[t] = make_float4((float)Z.x, (float)Z.y, (float)r2, r2 < 0x1p-100 ? 1.0f : 0.0f);
    }
    if (T == nullptr || Rs == nullptr || t >= ref_len * 16) return;
    const int k = t >> 4, d = t & 15;
    Fe32Bla r{0.0f, 0.0f, 0.0f, 0.0f, 0, 0, 0, 0};
    double rs = 0.0;
    if (d < levels) {
        const double* e = T + ((size_t)d * ref_len + k) * 5;
        rs = ldexp(e[4], kRadiusBias);
        split_pair(e[0], e[1], r.ar, r.ai, r.ea);
        split_pair(e[2], e[3], r.br, r.bi, r.eb);
    }
    Rs[t] = rs;
    AB[t] = r;
}

// One pixel per thread, blocks of 8x8 pixels (warps of 8x4): a block lives as long as
// its slowest pixel, so small blocks let an SM start new ones as each ends.
template <int FT, bool BLA, bool REBASE>
__global__ void __launch_bounds__(64, 16) fe32_coarse_kernel(const ApFrameParams p,
                                                             const ApFrameBuffers b) {
    const int i = blockIdx.x * 8 + (threadIdx.x & 7);
    const int j = blockIdx.y * 8 + (threadIdx.x >> 3);
    if (i >= p.width || j >= p.height) return;
    Fe32Run s;
    if (!fe32_begin(p, b, i, j, s)) return;
    fe32_advance<FT, BLA, REBASE, false>(p, b, s, 0);
    fe32_finish(p, b, s);
}

template <int FT>
static void launch_fe32_ft(const ApFrameParams& p, const ApFrameBuffers& b, bool bla, bool rebase,
                           cudaStream_t st) {
    const dim3 grid((p.width + 7) / 8, (p.height + 7) / 8);
    if (bla && rebase)
        fe32_coarse_kernel<FT, true, true><<<grid, 64, 0, st>>>(p, b);
    else if (bla)
        fe32_coarse_kernel<FT, true, false><<<grid, 64, 0, st>>>(p, b);
    else if (rebase)
        fe32_coarse_kernel<FT, false, true><<<grid, 64, 0, st>>>(p, b);
    else
        fe32_coarse_kernel<FT, false, false><<<grid, 64, 0, st>>>(p, b);
}

int launch_fe32(const ApFrameParams& p, const ApFrameBuffers& b, cudaStream_t st) {
    const bool bla = p.bla_levels > 1;
    if (p.tier != AP_TIER_FLOATEXP32)
        return AP_E_UNSUPPORTED;
    if (p.mode != AP_MODE_COARSE || !(p.flags & AP_FLAG_NO_RGB)) {
        set_error("AP_TIER_FLOATEXP32 serves coarse passes without in-kernel colour (set AP_FLAG_NO_RGB)");
        return AP_E_INVALID;
    }
    const int ft = p.fractal_type;
    const bool rebase = (p.flags & AP_FLAG_REBASE) != 0;
    if (ft < 0 || ft > 4) {
        set_error("AP_TIER_FLOATEXP32: fractal_type 0..4");
        return AP_E_INVALID;
    }
    if (rebase && (ft == 2 || ft == 3 || p.rebase_pass > 0 || p.ref_len < 1)) {
        set_error("AP_FLAG_REBASE serves fractal types 0, 1 and 4 in one pass (rebase_pass 0, ref_len >= 1)");
        return AP_E_UNSUPPORTED;
    }
    if (!b.orbit_packed || (bla && !b.bla_packed) || p.bla_levels > 16 || p.bbsa_skip > 0) {
        set_error("AP_TIER_FLOATEXP32 needs ap_pack_fe32 inputs (orbit_packed, bla_packed) and no series start");
        return AP_E_INVALID;
    }
    // the Burning Ship formulas take no leaps (as the FloatExp tier's reference kernels)
    if (ft == 0 || ft == 2)
        launch_fe32_ft<kFtQuad>(p, b, bla, rebase, st);
    else if (ft == 1 || ft == 3)
        launch_fe32_ft<kFtShip>(p, b, false, rebase, st);
    else
        launch_fe32_ft<kFtMulti>(p, b, bla, rebase, st);
    return check_launch("fe32_coarse_kernel");
}

}  // namespace ap

extern "C" int ap_pack_fe32(const double* orbit_packed, int32_t ref_len, const double* table,
                            int32_t levels, double* orbit32_out, double* bla_out, void* stream) {
    if (!orbit_packed || !orbit32_out || ref_len < 0 || (table && (!bla_out || levels < 1 ||
        levels > 16)) || (reinterpret_cast<uintptr_t>(orbit32_out) & 15u) ||
        (bla_out && (reinterpret_cast<uintptr_t>(bla_out) & 31u))) {
        ap::set_error("ap_pack_fe32: bad arguments");
        return AP_E_INVALID;
    }
    const int n = ref_len + 1;
    const int m = table ? ref_len * 16 : 0;
    const int total = n > m ? n : m;
    double* Rs = bla_out;
    ap::Fe32Bla* AB = bla_out ? reinterpret_cast<ap::Fe32Bla*>(bla_out + (size_t)ref_len * 16) : nullptr;
    ap::pack_fe32_kernel<<<(total + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const double4*>(orbit_packed), n, table, levels, ref_len,
        reinterpret_cast<float4*>(orbit32_out), Rs, AB);
    return ap::check_launch("pack_fe32_kernel");
}
