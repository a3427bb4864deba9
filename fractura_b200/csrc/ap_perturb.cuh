// ap_perturb.cuh -- perturbation tiers (FP64 deltas and FloatExp deltas).
#pragma once

#include "ap_common.cuh"

namespace ap {

template <int ARITH>
__device__ __forceinline__ SampleOut perturb_sample_at(const ApFrameParams& p,
                                                       const ApFrameBuffers& b, double sub_i,
                                                       double sub_j) {
    (void)p; (void)b; (void)sub_i; (void)sub_j;
    return interior_sample();
}

template <int ARITH>
__device__ __forceinline__ SampleOut floatexp_sample_at(const ApFrameParams& p,
                                                        const ApFrameBuffers& b, double sub_i,
                                                        double sub_j) {
    (void)p; (void)b; (void)sub_i; (void)sub_j;
    return interior_sample();
}

}  // namespace ap
