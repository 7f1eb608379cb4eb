// Instantiations for cuhc::CosineMetric, part core (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_CORE(cuhc::CosineMetric)
