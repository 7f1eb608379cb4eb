// Instantiations for cuhc::ChebyshevMetric, part core (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_CORE(cuhc::ChebyshevMetric)
