// Instantiations for cuhc::SqEuclideanMetric, part mst (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_MST(cuhc::SqEuclideanMetric)
