// Instantiations for cuhc::ChebyshevMetric (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_METRIC(cuhc::ChebyshevMetric)
