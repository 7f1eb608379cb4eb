// Instantiations for cuhc::ChebyshevMetric, part mst (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_MST(cuhc::ChebyshevMetric)
