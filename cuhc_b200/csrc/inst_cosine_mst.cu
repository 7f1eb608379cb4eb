// Instantiations for cuhc::CosineMetric, part mst (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_MST(cuhc::CosineMetric)
