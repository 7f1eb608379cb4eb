// Instantiations for cuhc::CosineMetric, part mreach (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_MREACH(cuhc::CosineMetric)
