// ap_peak.cu -- dependent-FMA throughput probe used as the roofline
// denominator of the iteration kernels (which are bound by the FP64 / FP32
// vector pipes, not by HBM or tensor cores).  Measurement helper; it has no
// counterpart in the reference.
#include "ap_common.cuh"

namespace ap {

constexpr int kChains = 8;

template <typename T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T* out, int iters, T a, T b) {
    T x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = (T)(threadIdx.x + c) * (T)1e-3;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == (T)-12345.0) out[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace ap

// precision: 64 or 32.  Launches blocks x 256 threads, each running 8 chains
// of `iters` dependent FMAs; *flops receives 2 * 8 * iters * threads.
extern "C" int ap_fma_peak_launch(int32_t precision, int32_t blocks, int32_t iters,
                                         void* scratch, double* flops, void* stream) {
    if (!scratch || !flops || blocks <= 0 || iters <= 0 || (precision != 64 && precision != 32)) {
        ap::set_error("ap_fma_peak_launch: bad arguments");
        return AP_E_INVALID;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (precision == 64)
        ap::fma_peak_kernel<double><<<blocks, 256, 0, st>>>(static_cast<double*>(scratch), iters,
                                                            0.999999999, 1e-9);
    else
        ap::fma_peak_kernel<float><<<blocks, 256, 0, st>>>(static_cast<float*>(scratch), iters,
                                                           0.9999999f, 1e-7f);
    *flops = 2.0 * ap::kChains * (double)iters * (double)blocks * 256.0;
    return ap::check_launch("fma_peak_kernel");
}
