// Instantiations for cuhc::EuclideanMetric, part mreach (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_MREACH(cuhc::EuclideanMetric)
