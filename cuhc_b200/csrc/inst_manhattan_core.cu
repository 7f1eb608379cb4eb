// Instantiations for cuhc::ManhattanMetric, part core (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_CORE(cuhc::ManhattanMetric)
