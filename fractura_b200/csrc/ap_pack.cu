// ap_pack.cu -- device re-layout of the reference orbit and the BLA table into
// the records the perturbation kernels read (one load per step, one 128-byte
// row per level search).  Values are copied or computed exactly as the
// per-step code computes them, so results do not change.
#include "ap_common.cuh"

namespace ap {

__global__ void __launch_bounds__(256) pack_orbit_kernel(const double* __restrict__ re,
                                                         const double* __restrict__ im, int n,
                                                         double4* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double rx = re[k], ry = im[k];
    const double r_mag2 = rx * rx + ry * ry;
    // Safe radius s: for |dz| < s the rounded |Z + dz|^2 is neither above the
    // bailout 65536 (|Z| + s <= 256 (1 - 1e-12)), nor below the Pauldelbrot
    // threshold 1e-6 |Z|^2, nor below the rounded |dz|^2 (the rebase test):
    // s <= |Z| (1 - 1e-7) / 2 keeps |Z + dz| >= |Z| - s > s (1 + 1e-7) > |dz|,
    // and 1e-6 |Z|^2 < s^2 covers the Pauldelbrot threshold.  The 1e-12 margins
    // cover the roundings of |Z|, of Z + dz and of the squares.  Stored as
    // s^2 (1 - 1e-12) to be compared with the rounded |dz|^2.
    const double rz = sqrt(r_mag2);
    double s = 256.0 * (1.0 - 1e-12) - rz * (1.0 + 1e-12);
    s = fmin(s, rz * (1.0 - 1e-12) * 0.5 * (1.0 - 1e-7));
    s = s > 0.0 ? s : 0.0;
    if (k == n - 1) s = 0.0;  // the orbit's end is never a safe step (the rebase kernels rely on it)
    // slot 3: the level-0 BLA radius, written by ap_pack_bla (0: no leap)
    out[k] = make_double4(rx, ry, s * s * (1.0 - 1e-12), 0.0);
}

__global__ void __launch_bounds__(256) pack_bla_kernel(const double* __restrict__ T, int levels,
                                                       int ref_len, double* __restrict__ R,
                                                       double4* __restrict__ AB,
                                                       double* __restrict__ orb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;  // one (k, d) pair per thread
    if (t >= ref_len * 16) return;
    const int k = t >> 4, d = t & 15;
    if (d < levels) {
        const double* e = T + ((size_t)d * ref_len + k) * 5;
        // a level is admissible only if its leap ends before the orbit does
        // (k + 2^d < ref_len); the coarse loop relies on 0 radii elsewhere
        R[t] = (k + (1 << d) < ref_len) ? e[4] : 0.0;
        if (d == 0 && orb) orb[4 * (size_t)k + 3] = R[t];  // the orbit record's level-0 radius
        AB[t] = make_double4(e[0], e[1], e[2], e[3]);
    } else {
        R[t] = 0.0;
        AB[t] = make_double4(0.0, 0.0, 0.0, 0.0);
    }
}

}  // namespace ap

extern "C" int ap_pack_orbit(const double* ref_re, const double* ref_im, int32_t ref_len,
                             double* out, void* stream) {
    if (!ref_re || !ref_im || !out || ref_len < 0 || (reinterpret_cast<uintptr_t>(out) & 31u)) {
        ap::set_error("ap_pack_orbit: bad arguments (out must be 32-byte aligned)");
        return AP_E_INVALID;
    }
    const int n = ref_len + 1;
    ap::pack_orbit_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        ref_re, ref_im, n, reinterpret_cast<double4*>(out));
    return ap::check_launch("pack_orbit_kernel");
}

extern "C" int ap_pack_bla(const double* table, int32_t levels, int32_t ref_len, double* out,
                           double* orbit_packed, void* stream) {
    if (!table || !out || levels < 1 || levels > 16 || ref_len < 1 ||
        (reinterpret_cast<uintptr_t>(out) & 31u)) {
        ap::set_error("ap_pack_bla: bad arguments (1 <= levels <= 16, out 32-byte aligned)");
        return AP_E_INVALID;
    }
    double* R = out;
    double4* AB = reinterpret_cast<double4*>(out + (size_t)ref_len * 16);
    const int n = ref_len * 16;
    ap::pack_bla_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        table, levels, ref_len, R, AB, orbit_packed);
    return ap::check_launch("pack_bla_kernel");
}
