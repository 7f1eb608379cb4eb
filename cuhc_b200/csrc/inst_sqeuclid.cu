// Instantiations for cuhc::SqEuclideanMetric (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_METRIC(cuhc::SqEuclideanMetric)
