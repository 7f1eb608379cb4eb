// Instantiations for cuhc::ManhattanMetric, part mst (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_MST(cuhc::ManhattanMetric)
