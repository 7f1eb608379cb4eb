// Instantiations for cuhc::MinkowskiMetric, part mst (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_MST(cuhc::MinkowskiMetric)
