// Instantiations for cuhc::CosineMetric (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_METRIC(cuhc::CosineMetric)
