// Exact minimum spanning tree by Borůvka rounds, entirely on the GPU, and
// the scipy-format merge tree built from it.
#pragma once

#include <vector>

#include "common.cuh"
#include "radius.cuh"
#include "spatial.cuh"

namespace cuhc {

// Counters of the passes of one call (exported by cuhc_prune_stats and the
// extended statistics call).
struct PassStats {
  unsigned long long tilesComputed = 0, tilesTotal = 0;
  unsigned long long passes = 0, rounds = 0;
};

// MST edges in original point indices (u < v), on the device.
struct DeviceEdges {
  DeviceBuffer<int> u, v;
  DeviceBuffer<float> w;
  int count = 0;
};

// Sorts MST edges by the reference's edge order (weight, u, v)
// (mst.cuh:41-48) on the device and copies them to the host.
int sortEdgesToHost(DeviceEdges &edges, int numEdges, cudaStream_t stream, std::vector<int> &u,
                    std::vector<int> &v, std::vector<float> &w);

// Sorted edges in page-locked host memory owned by the calling thread: the
// buffers grow as needed and are reused by the thread's next call, so a call
// pays neither page faults nor a staged copy. Valid until that next call.
struct HostEdges {
  const int *u = nullptr, *v = nullptr;
  const float *w = nullptr;
  int count = 0;
};
int sortEdgesToPinned(DeviceEdges &edges, int numEdges, cudaStream_t stream, HostEdges &out);
// Edges of a batch (original ids = rows of the concatenated points, instance
// i owning rows offsets[i] .. offsets[i + 1] - 1): sorted by (instance,
// weight, u, v) on the device, endpoints in each instance's local ids, into
// the same thread-owned page-locked buffers; counts[i] = instance i's edges.
int sortBatchEdgesToPinned(DeviceEdges &edges, int numEdges,
                           const std::vector<long long> &offsets, cudaStream_t stream,
                           HostEdges &out, std::vector<int> &counts);

// scipy linkage rows from merges in tree order (each merge after the merges
// that made its clusters): union-find names clusters, as the reference's
// treeFromOrderedMerges (mst.cuh:204-228). Z receives (n-1) x 4 doubles.
void treeFromOrderedMerges(const std::vector<int> &u, const std::vector<int> &v,
                           const std::vector<float> &w, int n, double *Z);
// The same over plain arrays of n - 1 merges.
void treeFromOrderedMerges(const int *u, const int *v, const float *w, int n, double *Z);

// Whether merges can form a tree: n-1 merges, finite heights, each joining
// two clusters not yet joined (mst.cuh:188-202).
bool mergesFormTree(const std::vector<int> &u, const std::vector<int> &v,
                    const std::vector<float> &w, int n);

// HDBSCAN's k-NN lists (a by-product of the core-distance pass), by
// position: the positions of each point's k nearest points in ascending
// distance (itself included) and a flag set when a point outside the list
// lies at exactly the k-th distance.
struct KnnLists {
  const int *pos = nullptr;
  const int *tie = nullptr;
  int k = 0;
};

// Borůvka over the points of an index (Metric x Weight instantiations in
// inst_<metric>_mst.cu and inst_<metric>_mreach.cu). Fills edges with the
// n-1 MST edges (original indices).
// With knn (mutual reachability, alpha 1), every round first seeds each row
// with its lightest list edge to another component and settles the rows
// whose list edge is provably their answer (boruvka.cuh, seedFromKnn).
template <class Metric, class Weight>
int boruvkaMst(SpatialIndex &index, const Metric &metric, const Weight &weight, bool prune,
               DeviceEdges &edges, PassStats *stats, cudaStream_t stream,
               RadiusLog *radiusLog = nullptr, const KnnLists *knn = nullptr);

// Exact core distances (k-th nearest, the point itself first) by position;
// with knnPos / knnTie (n x k and n ints) also the k-NN lists (KnnLists).
template <class Metric>
int coreDistances(SpatialIndex &index, const Metric &metric, int k, bool prune, float *core,
                  PassStats *stats, cudaStream_t stream, const int *coreRank = nullptr,
                  int *knnPos = nullptr, int *knnTie = nullptr);

// The same core distances for any 1 <= k <= n by radix select over chunks of
// the materialised distance matrix (radix.cuh). Bit-identical to
// coreDistances.
template <class Metric> bool screenable(SpatialIndex &index, int k);

template <class Metric>
float timeKnnSample(SpatialIndex &index, const Metric &metric, int k, bool screened,
                    int sampleTiles, float *core, cudaStream_t stream);

template <class Metric>
int coreDistancesRadix(SpatialIndex &index, const Metric &metric, int k, float *core,
                       cudaStream_t stream);

} // namespace cuhc
