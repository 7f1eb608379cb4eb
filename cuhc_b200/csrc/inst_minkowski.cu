// Instantiations for cuhc::MinkowskiMetric (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_METRIC(cuhc::MinkowskiMetric)
