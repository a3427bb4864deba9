// ap_tiers.cuh -- sample evaluators of the non-FP64 tiers.
#pragma once

#include "ap_dd.cuh"
#include "ap_perturb.cuh"
