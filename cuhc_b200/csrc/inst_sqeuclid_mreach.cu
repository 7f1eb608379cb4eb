// Instantiations for cuhc::SqEuclideanMetric, part mreach (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_MREACH(cuhc::SqEuclideanMetric)
