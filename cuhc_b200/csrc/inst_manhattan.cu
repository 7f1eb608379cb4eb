// Instantiations for cuhc::ManhattanMetric (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_METRIC(cuhc::ManhattanMetric)
