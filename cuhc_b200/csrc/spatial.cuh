// Spatial index of a point set on the GPU: k-d order, tiled layout, BVH.
//
//  order     the k-d order: position p holds original point order[p]. Each
//            range is split at a tile boundary near its middle (left side:
//            floor(tiles / 2) tiles) along the feature with the widest
//            spread of a sample, as the reference's spatialOrder does
//            (spatial.cuh:44-91), but built on the GPU one tree level at a
//            time with a radix sort per level instead of a CPU nth_element.
//            Results never depend on the order: every pass breaks ties by
//            original index.
//  tiled     the points in HBM in the engine's layout: tile t, feature
//            chunk c is a contiguous [KC][128] block (feature-major, zero
//            padded), so one tile chunk is a single 16-byte-aligned copy of
//            KC * 512 bytes straight into shared memory in the order the
//            distance loop reads it.
//  BVH       the balanced binary tree of the split: node = range of tiles,
//            leaves = tiles. Every node has a bounding box; per pass each
//            node also carries its smallest per-point value (core distance
//            or cluster size) and its component if all its points share one.
#pragma once

#include <vector>

#include "common.cuh"

namespace cuhc {

struct BvhTopology {
  int numNodes = 0, numTiles = 0, depth = 0;
  // Host copies (breadth-first node order: parents before children, each
  // level left to right, so every level is a contiguous node range).
  std::vector<int> left, right, firstTile, tileCount, levelStart;
  std::vector<int> leafOfTile;
  std::vector<unsigned char> spans; // node holds tiles of several instances
  std::vector<int> rootOfInstance;  // node whose tiles are exactly the instance's
  // One instance: balanced halves (left child floor(count / 2) tiles).
  void build(int numTiles);
  // Consecutive instances of instanceTiles[i] tiles each: a node holding
  // several instances splits at the instance boundary nearest its middle
  // tile; inside an instance, balanced halves as in build().
  void buildForest(const std::vector<int> &instanceTiles);
};

struct SpatialIndex {
  int n = 0, d = 0, numTiles = 0, kc = 0, numChunks = 0;
  cudaStream_t stream = 0;
  BvhTopology topo;
  DeviceBuffer<float> tiled;         // numTiles * numChunks * kc * 128
  DeviceBuffer<int> order, rank;     // position -> original, original -> position
  DeviceBuffer<int> nodeLeft, nodeRight, nodeFirstTile, nodeTileCount, leafOfTile;
  DeviceBuffer<float> nodeLow, nodeHigh; // numNodes * d
  DeviceBuffer<float> nodeMinValue;      // numNodes
  DeviceBuffer<int> nodePure;            // numNodes: component if pure, else -1
  bool hasMinValues = false;             // nodeMinValue filled by updateMinValues
  // Batches of instances (buildBatch): each instance starts on a fresh tile;
  // the slots after its last point are padding (order == -1). n counts every
  // position then, padding included.
  int numInstances = 1, numPads = 0, numPoints = 0;
  std::vector<int> instanceFirstTile;    // host, per instance
  DeviceBuffer<int> rootOfTile;          // traversal root per tile (batches)
  DeviceBuffer<unsigned char> nodeSpans; // batches
  // Heavy-first launch order of the passes (orderTiles).
  DeviceBuffer<unsigned int> tileWork;   // column tiles each row tile computed last pass
  DeviceBuffer<int> tileOrder;           // row tiles, heaviest first
  DeviceBuffer<unsigned int> tileKeys, tileKeysSorted;
  DeviceBuffer<int> tileIota;
  DeviceBuffer<unsigned char> tileSortTemp;
  size_t tileSortBytes = 0;
  bool tileWorkValid = false;            // a pass has recorded tileWork

  size_t tileFloats() const { return (size_t)numChunks * kc * kTile; }

  // Builds everything from points (n x d row-major, original order, device).
  // spatial=false keeps the original order (positions == original indices).
  int build(const float *points, int n, int d, bool spatial, cudaStream_t stream);
  // Builds one index over a batch of instances: sizes[i] consecutive rows of
  // points each (original order), every instance its own k-d tree and BVH
  // subtree (rootOfTile), so traversals never leave their instance.
  int buildBatch(const float *points, const std::vector<int> &sizes, int d,
                 cudaStream_t stream);
  int buildCommon(const float *points, int positions, int d, bool spatial,
                  const std::vector<int> *hostOrder, cudaStream_t stream);
  // Re-tiles new point data already in position order (RNN centroids after a
  // round), keeping the order arrays; recomputes boxes.
  int retile(const float *pointsByPosition, int n);
  // Per-node smallest value of values[position] (null: all zero).
  int updateMinValues(const float *valuesByPosition);
  // Per-node purity of component[position] (null: every node impure).
  int updatePurity(const int *componentByPosition);
  // Whether every coordinate's extent over all points (the root box) is
  // finite and at most `limit`. Copies the root box to the host and waits
  // for the index stream.
  bool extentsWithin(float limit);
  // Whether every point's squared norm is 0 or within [low, high] (the
  // cosine screen's range). Computed once per index; retile resets it.
  bool normsWithin(float low, float high);
  bool normRangeKnown = false;
  float normLow = 0.0f, normHigh = 0.0f;
  // tileOrder <- row tiles by decreasing tileWork (fromBoxes: by decreasing
  // leaf box log-volume, the estimate before any pass has run). Enqueued on
  // the index stream with no host work (buffers are allocated on first use).
  // impureFirst: row tiles whose points span several components (nodePure
  // of the round) go before the others, each group heaviest first.
  int orderTiles(bool fromBoxes, bool impureFirst = false);
};

} // namespace cuhc
