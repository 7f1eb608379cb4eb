// Instantiations for cuhc::EuclideanMetric (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_METRIC(cuhc::EuclideanMetric)
