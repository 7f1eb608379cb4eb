// Instantiations for cuhc::EuclideanMetric, part core (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_CORE(cuhc::EuclideanMetric)
