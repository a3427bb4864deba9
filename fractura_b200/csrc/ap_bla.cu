// ap_bla.cu -- chained bilinear-approximation table built on the device.
#include "ap_common.cuh"

extern "C" int ap_build_bla(const double* ref_re, const double* ref_im, int32_t ref_len,
                            int32_t fractal_type, double tol, int32_t levels, int32_t gen_n,
                            double gen_kr, double gen_ki, double* out, void* stream) {
    (void)ref_re; (void)ref_im; (void)ref_len; (void)fractal_type; (void)tol; (void)levels;
    (void)gen_n; (void)gen_kr; (void)gen_ki; (void)out; (void)stream;
    ap::set_error("ap_build_bla: not built yet");
    return AP_E_UNSUPPORTED;
}
