// Ward linkage: RNN rounds, NN-chain, dense Lance-Williams (see rnn.cuh).
#include "rnn.cuh"

namespace cuhc {

int rnnWard(const float *, int, int, const RnnOptions &, double *, PassStats *, cudaStream_t) {
  return kErrorInvalidAlgorithm;
}

int nnChainWard(const float *, int, int, double *, cudaStream_t) { return kErrorInvalidAlgorithm; }

int denseLinkage(const float *, int, int, int, float, int, double *, cudaStream_t) {
  return kErrorInvalidAlgorithm;
}

} // namespace cuhc
