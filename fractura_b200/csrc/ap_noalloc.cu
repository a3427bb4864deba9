// ap_noalloc.cu -- histogram -> CDF for callers that cannot allocate device memory.
//
// ap_histogram_cdf needs a num_bins int32 scratch histogram from its caller.
// Some callers cannot provide one: code that runs where cudaMalloc is not
// allowed or not wanted (inside a host callback, a real-time render loop that
// must not hit the allocator, or a plugin whose host owns every allocation).
// ap_histogram_cdf_noalloc serves them from a fixed array compiled into this
// library instead.  The array lives in every GPU's global memory from the
// moment the library's module is loaded on that GPU until the process exits.
#include <mutex>

#include "ap_common.cuh"

namespace ap {

constexpr int kNoAllocMaxBins = AP_NOALLOC_MAX_BINS;
constexpr int kMaxDevices = 64;

// The histogram scratch shared by every call on a device (256 KiB).
static __device__ __align__(256) int32_t g_noalloc_hist[kNoAllocMaxBins];

// Device address of g_noalloc_hist per device, looked up once.  The name
// g_noalloc_hist in host code is only a host-side stand-in, so the address
// has to come from cudaGetSymbolAddress with the device current.  A device reset
// reloads the module and makes the kept address stale; the header says so.
static int32_t* g_noalloc_ptr[kMaxDevices] = {};
static std::mutex g_noalloc_mu;

static int noalloc_scratch(int32_t** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_error("ap_histogram_cdf_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
        return AP_E_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("ap_histogram_cdf_noalloc: device %d outside 0..%d", dev, kMaxDevices - 1);
        return AP_E_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_ptr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_hist);
        if (e != cudaSuccess || p == nullptr) {
            set_error("ap_histogram_cdf_noalloc: cudaGetSymbolAddress: %s",
                      cudaGetErrorString(e));
            return AP_E_CUDA;
        }
        g_noalloc_ptr[dev] = static_cast<int32_t*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return AP_OK;
}

}  // namespace ap

extern "C" int ap_histogram_cdf_noalloc(const float* iter_map, int32_t width, int32_t height,
                                        int32_t max_iter, int32_t num_bins, float* cdf,
                                        void* stream) {
    if (num_bins < 2 || num_bins > ap::kNoAllocMaxBins) {
        ap::set_error("ap_histogram_cdf_noalloc: num_bins %d outside 2..%d (the built-in scratch "
                      "holds %d bins)", num_bins, ap::kNoAllocMaxBins, ap::kNoAllocMaxBins);
        return AP_E_INVALID;
    }
    int32_t* hist = nullptr;
    const int rc = ap::noalloc_scratch(&hist);
    if (rc != AP_OK) return rc;
    // The existing path, with the built-in array as its scratch; it clears the
    // bins it uses with cudaMemsetAsync before counting.
    return ap_histogram_cdf(iter_map, width, height, max_iter, num_bins, hist, cdf, stream);
}
