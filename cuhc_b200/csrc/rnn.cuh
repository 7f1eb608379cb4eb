// Ward linkage (RNN rounds, NN-chain), dense Lance-Williams linkage, and the
// HDBSCAN condensed tree.
#pragma once

#include "mst.cuh"

namespace cuhc {

// Hand-over settings of the RNN rounds; the reference's RnnOptions
// (rnn_ward.cuh:66-86) with the same defaults.
struct RnnOptions {
  float minProgress = 0.01f;
  int denseBelow = 0;
  bool allowDense = true;
};

// Ward merge tree by rounds of reciprocal nearest neighbours on device points
// (original order); tree to the host. Bit-identical selection weights to the
// reference (fast division), exact heights and centroids in its formulas.
int rnnWard(const float *devPoints, int n, int d, const RnnOptions &options, double *hostTree,
            PassStats *stats, cudaStream_t stream);

// Ward by the nearest-neighbour chain.
int nnChainWard(const float *devPoints, int n, int d, double *hostTree, cudaStream_t stream);

// Any linkage on the dense n x n float32 matrix (Lance-Williams updates).
int denseLinkage(const float *devPoints, int n, int d, int metricId, float p, int linkageId,
                 double *hostTree, cudaStream_t stream);

// The pruning mode set by cuhc_set_pruning (0 auto, 1 always, 2 never).
int currentPruneMode();

// HDBSCAN's condensed tree of a (n-1) x 4 single-linkage tree (host):
// rows in sklearn 1.9's order; returns the row count, or -(rows needed) if
// capacity is too small.
long long condenseTree(const double *tree, long long n, long long minClusterSize,
                       long long capacity, long long *parent, long long *child, double *lambda,
                       long long *size);

} // namespace cuhc
