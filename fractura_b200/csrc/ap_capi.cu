// ap_capi.cu -- error reporting and identity entry points of the C ABI.
#include <cstdarg>
#include <cstdio>

#include "ap_common.cuh"

namespace ap {

static thread_local char g_last_error[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap_list;
    va_start(ap_list, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap_list);
    va_end(ap_list);
}

static unsigned long long g_launches = 0;

int check_launch(const char* what) {
    __atomic_fetch_add(&g_launches, 1ULL, __ATOMIC_RELAXED);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return AP_E_CUDA;
    }
    return AP_OK;
}

}  // namespace ap

extern "C" int ap_abi_version(void) { return AP_ABI_VERSION; }

extern "C" const char* ap_last_error(void) { return ap::g_last_error; }

extern "C" uint64_t ap_launch_counter(void) {
    return __atomic_load_n(&ap::g_launches, __ATOMIC_RELAXED);
}
