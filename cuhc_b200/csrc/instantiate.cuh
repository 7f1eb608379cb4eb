// Explicit instantiation of the per-metric entry points. One translation
// unit per metric family (inst_*.cu) so that the builds run in parallel.
#pragma once

#include "boruvka.cuh"
#include "pairwise.cuh"
#include "radix.cuh"

namespace cuhc {

template <class Metric>
int pairwiseDistances(const float *A, int nA, const float *B, int nB, int d, const Metric &m,
                      float *out, cudaStream_t s) {
  DeviceBuffer<float> tiledA, tiledB;
  StatusChain st;
  CUHC_TRY(st, buildTiled(A, nA, d, tiledA, s));
  if (B)
    CUHC_TRY(st, buildTiled(B, nB, d, tiledB, s));
  CUHC_TRY(st, launchPairwise(tiledA.get(), B ? tiledB.get() : tiledA.get(), nA, nB, d, m, out, s));
  CUHC_TRY(st, cudaStreamSynchronize(s));
  return st.code;
}

} // namespace cuhc

// Three parts per metric, one translation unit each (inst_<metric>_<part>.cu),
// so that the slowest metric (minkowski: exp2f / log2f per pair in every
// kernel) does not serialise the build.
#define CUHC_INSTANTIATE_MST(M)                                                                    \
  template int cuhc::boruvkaMst<M, cuhc::PlainWeight>(                                             \
      cuhc::SpatialIndex &, const M &, const cuhc::PlainWeight &, bool, cuhc::DeviceEdges &,       \
      cuhc::PassStats *, cudaStream_t, cuhc::RadiusLog *, const cuhc::KnnLists *);

#define CUHC_INSTANTIATE_MREACH(M)                                                                 \
  template int cuhc::boruvkaMst<M, cuhc::MutualReachWeight>(                                       \
      cuhc::SpatialIndex &, const M &, const cuhc::MutualReachWeight &, bool, cuhc::DeviceEdges &, \
      cuhc::PassStats *, cudaStream_t, cuhc::RadiusLog *, const cuhc::KnnLists *);

#define CUHC_INSTANTIATE_CORE(M)                                                                   \
  template int cuhc::coreDistances<M>(cuhc::SpatialIndex &, const M &, int, bool, float *,         \
                                      cuhc::PassStats *, cudaStream_t, const int *, int *, int *); \
  template bool cuhc::screenable<M>(cuhc::SpatialIndex &, int);                                    \
  template float cuhc::timeKnnSample<M>(cuhc::SpatialIndex &, const M &, int, bool, int, float *,  \
                                        cudaStream_t);                                             \
  template int cuhc::coreDistancesRadix<M>(cuhc::SpatialIndex &, const M &, int, float *,          \
                                           cudaStream_t);                                          \
  template int cuhc::pairwiseDistances<M>(const float *, int, const float *, int, int, const M &,  \
                                          float *, cudaStream_t);
