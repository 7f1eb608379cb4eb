// The exact FP32 distance engine and the two all-pairs passes built on it.
//
// Block shape: 256 threads own one ROW TILE of 128 points for the whole
// pass. Thread (tr, tc) = (tid / 16, tid % 16) computes an 8 x 8 register
// block of pairs: rows tr*4+{0..3} and 64+tr*4+{0..3}, columns likewise with
// tc. The 16 threads that share a row are one half-warp, so a row's results
// are owned by exactly one half-warp and need no atomics.
//
// Per column tile the block stages the tile's features in shared memory,
// chunk by chunk (KC features x 128 points, feature-major, one contiguous
// copy from the tiled HBM layout), and folds each feature into the 64
// accumulators: metric.accumulate(acc, row value, column value), features in
// order 0..d-1, the reference's operation order (distance_matrix.cuh:
// 108-175), so every distance is bit-identical to the reference's.
//
// What differs from the reference is the epilogue and the tile schedule:
//
//  * Filtered epilogue. Each row keeps a filter bound derived from its
//    current threshold (best edge so far, or the k-th distance so far). The
//    fast path only takes a masked minimum of the filter values per row;
//    exact weights, sqrt and key compares run only when some pair of the
//    warp can still win. Winners are chosen by the exact packed key
//    (weight bits, ORIGINAL index), ties to the lower index.
//
//  * Nearest-first BVH traversal. Warp 0 walks the tile tree depth first,
//    nearer child first, and prunes a subtree when a lower bound of every
//    edge into it exceeds the largest threshold of the block's rows
//    (strictly: a pruned pair can not even tie). In Borůvka passes the row
//    threshold is min(row best, component best): an edge heavier than the
//    best edge already known to leave the row's component can not be that
//    component's minimum, so large components stop searching early. Subtrees
//    whose points all share the row tile's (single) component are skipped.
#pragma once

#include "common.cuh"
#include "metrics.cuh"
#include "spatial.cuh"

namespace cuhc {

constexpr int kThreads = 256;
constexpr int kStackSize = 96;

struct TileGeom {
  int tr, tc;
  __device__ __forceinline__ TileGeom() : tr(threadIdx.x >> 4), tc(threadIdx.x & 15) {}
  __device__ __forceinline__ int row(int r) const { return r < 4 ? tr * 4 + r : 60 + tr * 4 + r; }
  __device__ __forceinline__ int col(int c) const { return c < 4 ? tc * 4 + c : 60 + tc * 4 + c; }
};

// Folds KC features of a staged chunk into the 8 x 8 accumulators.
template <class Metric, int KC>
__device__ __forceinline__ void accumulateChunk(const float *__restrict__ sA,
                                                const float *__restrict__ sB, const Metric &m,
                                                typename Metric::Acc (&acc)[8][8],
                                                const TileGeom &g) {
#pragma unroll
  for (int k = 0; k < KC; ++k) {
    const float4 a0 = reinterpret_cast<const float4 *>(sA + k * kTile)[g.tr];
    const float4 a1 = reinterpret_cast<const float4 *>(sA + k * kTile + 64)[g.tr];
    const float4 b0 = reinterpret_cast<const float4 *>(sB + k * kTile)[g.tc];
    const float4 b1 = reinterpret_cast<const float4 *>(sB + k * kTile + 64)[g.tc];
    const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
    const float b[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
    if constexpr (Metric::kPacked) {
      // Two adjacent columns per packed instruction.
      const float2 b2[4] = {make_float2(b[0], b[1]), make_float2(b[2], b[3]),
                            make_float2(b[4], b[5]), make_float2(b[6], b[7])};
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const float2 negA = make_float2(-a[r], -a[r]);
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const float2 s = m.accumulate2(make_float2(acc[r][2 * c], acc[r][2 * c + 1]), negA, b2[c]);
          acc[r][2 * c] = s.x;
          acc[r][2 * c + 1] = s.y;
        }
      }
    } else {
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int c = 0; c < 8; ++c)
          acc[r][c] = m.accumulate(acc[r][c], a[r], b[c]);
    }
  }
}

__device__ __forceinline__ void copyChunk(float *__restrict__ dst, const float *__restrict__ src,
                                          int floats) {
  const float4 *s = reinterpret_cast<const float4 *>(src);
  float4 *t = reinterpret_cast<float4 *>(dst);
  for (int i = threadIdx.x; i < floats / 4; i += kThreads)
    t[i] = __ldg(s + i);
}

// Accumulators of the pairs (row tile I, column tile J). sA holds row tile
// chunk 0 when numChunks == 1 (then it stays resident for the whole pass).
// tiledA / tiledB may be the same array (a pass) or two (pairwise matrix);
// sA is only reloaded when the tile has several chunks.
template <class Metric, int KC>
__device__ __forceinline__ void computeTile(const float *__restrict__ tiledA,
                                            const float *__restrict__ tiledB, int numChunks,
                                            int tileI, int tileJ, float *sA, float *sB,
                                            const Metric &m, typename Metric::Acc (&acc)[8][8],
                                            const TileGeom &g) {
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c)
      acc[r][c] = m.init();
  const size_t tileFloats = (size_t)numChunks * KC * kTile;
  for (int chunk = 0; chunk < numChunks; ++chunk) {
    const float *srcA = tiledA + tileI * tileFloats + (size_t)chunk * KC * kTile;
    const float *srcB = tiledB + tileJ * tileFloats + (size_t)chunk * KC * kTile;
    if (numChunks > 1)
      copyChunk(sA, srcA, KC * kTile);
    const bool selfResident = numChunks == 1 && tileI == tileJ && tiledA == tiledB;
    if (!selfResident)
      copyChunk(sB, srcB, KC * kTile);
    __syncthreads();
    accumulateChunk<Metric, KC>(sA, selfResident ? sA : sB, m, acc, g);
    __syncthreads();
  }
}

// Shared state of a pass block besides the feature chunks.
struct PassShared {
  unsigned long long rowBest[kTile];
  float rowFilter[kTile];
  float rowThr[kTile];
  int colComp[kTile];
  float colValue[kTile];
  int colOrig[kTile];
  int stackNode[kStackSize];
  float stackLb[kStackSize];
  float warpMax[kThreads / 32];
  float thrTile;
  int sp;
  int next;
  int overflow;
};

struct PassParams {
  const float *tiled;
  int n, d, numChunks, numTiles;
  const int *order;     // position -> original index
  const int *component; // position -> component label (null: none)
  const int *nodeLeft, *nodeRight, *nodeFirstTile, *leafOfTile, *nodePure;
  const float *nodeLow, *nodeHigh, *nodeMinValue;
  bool prune;
  bool singletons;                // every point its own component (first round)
  unsigned long long *nearest;    // nearest-mode output, by position
  unsigned int *compBest;         // float bits by component label (null: none)
  float *core;                    // knn-mode output, by position
  int k;                          // knn-mode rank
  unsigned long long *tilesComputed;
  int *error;
  unsigned long long *screenStats; // ScreenCounter sums (null: not counted)
  unsigned long long *screenAudit; // ScreenAuditWord words (null: no audit)
  const int *rootOfTile;  // traversal root per row tile (null: node 0)
  const int *coreRank;    // knn-mode rank per position, 0 = core 0 (null: k for all)
  // Nearest mode: per-position cap on the row threshold (a proposed radius);
  // a negative value marks a row that is already settled: it neither
  // searches nor writes. Null: no cap.
  const float *radius;
  // Block b takes row tile tileOrder[b] (null: b), so that the heaviest row
  // tiles start first; tileWork[I] receives the column tiles row tile I
  // computed (null: not recorded).
  const int *tileOrder;
  unsigned int *tileWork;
  // Knn mode: per position, the positions of its k list entries in
  // ascending distance (k ints) and a flag set when a point outside the list
  // lies at exactly the k-th distance (null: not recorded).
  int *knnPos;
  int *knnTie;
  // Nearest mode: per position an initial best key (a real edge of the row,
  // kEmptyKey: none); kSettledKey in the index bits marks a key that is
  // already the row's answer: the row neither searches nor writes (null:
  // no seeds).
  const unsigned long long *seedKey;
  // Screened passes: per tile, the original indices, component labels and
  // weight values of its 128 slots packed as [3][128] 32-bit words, so that
  // one bulk copy stages a column tile's metadata (null: three copies from
  // order, component and the weight's value array).
  const int *packedMeta;
};

// Index bit of a seed key whose row is settled (indices stay below 2^30).
constexpr unsigned long long kSettledKey = 1ull << 31;

// Lower bound of every distance between the row tile box (shared memory)
// and a node box, by warp 0 (lanes split the features).
template <class Metric>
__device__ __forceinline__ float boxDistanceLowerBound(const Metric &m, const float *rowLow,
                                                       const float *rowHigh,
                                                       const float *nodeLow,
                                                       const float *nodeHigh, int d, int lane) {
  typename Metric::Acc acc = m.init();
  for (int f = lane; f < d; f += 32) {
    const float gap = fmaxf(0.0f, fmaxf(nodeLow[f] - rowHigh[f], rowLow[f] - nodeHigh[f]));
    acc = m.accumulate(acc, gap, 0.0f);
  }
  if constexpr (sizeof(typename Metric::Acc) == sizeof(float)) {
    for (int off = 16; off > 0; off /= 2)
      acc = m.combine(acc, __shfl_xor_sync(0xffffffffu, acc, off));
    return m.finalize(acc);
  } else {
    return 0.0f;
  }
}

// Warp 0: pops until it finds the next leaf (column tile) worth computing,
// or the stack runs dry (-1). Result in sh.next; the caller synchronizes.
template <class Metric, class Weight>
__device__ void traverseNext(const PassParams &p, const Metric &m, const Weight &w,
                             PassShared &sh, const float *rowLow, const float *rowHigh,
                             int rowTile, int rowPure, float rowMinValue, float slack) {
  const int lane = threadIdx.x & 31;
  int result = -1;
  while (true) {
    const int sp = sh.sp;
    if (sp == 0)
      break;
    const int node = sh.stackNode[sp - 1];
    const float lb = sh.stackLb[sp - 1];
    __syncwarp();
    if (lane == 0)
      sh.sp = sp - 1;
    __syncwarp();
    const float thr = sh.thrTile;
    if (lb > thr)
      continue;
    const int left = p.nodeLeft[node];
    if (left < 0) {
      const int tile = p.nodeFirstTile[node];
      if (tile == rowTile)
        continue;
      result = tile;
      break;
    }
    const int right = p.nodeRight[node];
    float lbChild[2];
    int child[2] = {left, right};
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int c = child[i];
      const int pure = p.nodePure ? p.nodePure[c] : -1;
      if (rowPure >= 0 && pure == rowPure) {
        lbChild[i] = INFINITY; // same single component: no edge inside
      } else if (p.prune && Metric::kBoxBound) {
        const float dlb = boxDistanceLowerBound(m, rowLow, rowHigh, p.nodeLow + (size_t)c * p.d,
                                                p.nodeHigh + (size_t)c * p.d, p.d, lane);
        const float v = p.nodeMinValue ? p.nodeMinValue[c] : 0.0f;
        lbChild[i] = w.lowerBound(dlb, rowMinValue, v) * slack;
      } else {
        lbChild[i] = 0.0f;
      }
    }
    // Push the farther child first so the nearer one is visited first.
    const int first = lbChild[0] <= lbChild[1] ? 1 : 0;
    if (lane == 0) {
      int s = sh.sp;
      for (int j = 0; j < 2; ++j) {
        const int i = j == 0 ? first : 1 - first;
        if (lbChild[i] <= thr && lbChild[i] < INFINITY) {
          if (s < kStackSize) {
            sh.stackNode[s] = child[i];
            sh.stackLb[s] = lbChild[i];
            ++s;
          } else {
            sh.overflow = 1;
          }
        }
      }
      sh.sp = s;
    }
    __syncwarp();
  }
  if (lane == 0)
    sh.next = result;
}

} // namespace cuhc
