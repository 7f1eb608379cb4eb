// Instantiations for cuhc::EuclideanMetric, part mst (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_MST(cuhc::EuclideanMetric)
