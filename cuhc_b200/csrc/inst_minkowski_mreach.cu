// Instantiations for cuhc::MinkowskiMetric, part mreach (see instantiate.cuh).
#include "instantiate.cuh"

CUHC_INSTANTIATE_MREACH(cuhc::MinkowskiMetric)
