// Instantiations for cuhc::ChebyshevMetric, part mreach (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_MREACH(cuhc::ChebyshevMetric)
