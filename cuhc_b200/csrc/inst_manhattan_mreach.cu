// Instantiations for cuhc::ManhattanMetric, part mreach (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_MREACH(cuhc::ManhattanMetric)
