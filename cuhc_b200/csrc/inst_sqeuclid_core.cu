// Instantiations for cuhc::SqEuclideanMetric, part core (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_CORE(cuhc::SqEuclideanMetric)
