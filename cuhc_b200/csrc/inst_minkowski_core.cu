// Instantiations for cuhc::MinkowskiMetric, part core (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_CORE(cuhc::MinkowskiMetric)
