// The all-pairs pass kernel (see engine.cuh for the block shape), in two
// modes:
//
//   nearest  for every point, its minimum-weight edge to a point of another
//            component, key (weight bits, original index): the Borůvka step
//            (single linkage, HDBSCAN) and the RNN-Ward nearest-cluster step
//            (every slot its own component). Same result as the reference's
//            nearestOtherComponent{,Symmetric,Walk}Kernel
//            (distance_matrix.cuh:228-390, spatial.cuh:215-343) for every row
//            whose component can still win; rows of a component whose best
//            edge is known to be lighter may stop early, which never changes
//            the component minimum.
//   knn      for every point, the k-th smallest distance with the point
//            itself counted as 0 (HDBSCAN core distances); the values of the
//            reference's kthNearestFusedKernel (hdbscan.cuh:144-258).
//
// Schedule of a block (one row tile):
//   1. the row tile against itself (seeds every row's threshold);
//   2. warp 0 collects candidate column tiles: it pops up to 32 BVH nodes at
//      a time from a shared frontier, one node per lane, tests each node's
//      weight lower bound against the block threshold, and appends surviving
//      leaves to a shared candidate list (up to kListCap per batch);
//   3. the list is sorted by lower bound (bitonic, in shared memory), so the
//      tiles are visited nearest first and thresholds tighten early;
//   4. the tiles are computed in that order. While tile i is computed, the
//      tensor memory accelerator copies tile i+1 (its feature block and its
//      original-index / component / value rows) into the other half of a
//      double buffer (cp.async.bulk on an mbarrier); a candidate whose bound
//      now exceeds the tightened threshold is skipped;
//   5. repeat from 2 until the frontier is empty.
#pragma once

#include "asyncload.cuh"
#include "engine.cuh"
#include "profiling.cuh"

namespace cuhc {

constexpr int kListCap = 1024;
// Flag on a candidate's tile index: all its points share one component.
constexpr int kPureColumnTile = 1 << 30;
// The frontier is a stack popped 32 at a time, each pop pushing at most two
// children one level deeper: it holds at most ~64 nodes per tree level, and
// the tile tree of 2^31 points is 24 levels deep. A full frontier stops the
// pass with an error (never a hang).
constexpr int kFrontierCap = 2048;

// Shared state of a pass block besides the staged tiles.
struct PassState {
  unsigned long long rowBest[kTile];
  float rowFilter[kTile];
  float warpMax[kThreads / 32];
  int listTile[kListCap];
  float listLb[kListCap];
  int frontNode[kFrontierCap];
  int rowTie[kTile]; // knn mode: a point outside the row's list ties its k-th value
  uint64_t bar[2];
  float thrTile;
  int listLen, frontLen, overflow;
};

// Column metadata of a staged tile (bulk-copy destinations, 512 B each).
struct ColumnMeta {
  int *orig;
  int *comp;
  float *value;
};

// Threads 0..127 (one row each) refresh the row filters and the block
// threshold; everyone must call it (it synchronizes).
template <class Metric, class Weight, bool kKnn>
__device__ __forceinline__ void refreshThresholds(const PassParams &p, const Metric &m,
                                                  const Weight &w, PassState &sh,
                                                  const float *lists, int firstRow) {
  const int tid = threadIdx.x;
  float t = -INFINITY;
  if (tid < kTile) {
    const int pos = firstRow + tid;
    // Padding slots and settled rows never search.
    const bool valid = pos < p.n && p.order[pos] >= 0 &&
                       !(!kKnn && p.seedKey && (p.seedKey[pos] & kSettledKey) &&
                         p.seedKey[pos] != kEmptyKey);
    float thr, filter = -INFINITY;
    if (kKnn) {
      thr = lists[tid * p.k + p.k - 1];
      if (valid)
        filter = m.filterBound(thr);
    } else {
      const unsigned long long key = sh.rowBest[tid];
      thr = key == kEmptyKey ? INFINITY : keyWeight(key);
      if (valid && p.compBest) {
        unsigned int *slot = p.compBest + p.component[pos];
        unsigned int cb = __ldcg(slot);
        if (key != kEmptyKey && floatBits(thr) < cb)
          cb = min(cb, atomicMin(slot, floatBits(thr)));
        thr = fminf(thr, bitsFloat(cb));
      }
      // A proposed radius caps the threshold after the component exchange
      // (only real edge weights go into compBest); negative: settled row.
      if (valid && p.radius)
        thr = fminf(thr, p.radius[pos]);
      const float v = valid ? w.load(pos) : 0.0f;
      if (valid && thr >= 0.0f && w.feasible(thr, v))
        filter = m.filterBound(w.distBound(thr, v));
    }
    sh.rowFilter[tid] = filter;
    t = filter == -INFINITY ? -INFINITY : thr;
  }
  for (int off = 16; off > 0; off /= 2)
    t = fmaxf(t, __shfl_xor_sync(0xffffffffu, t, off));
  if ((tid & 31) == 0)
    sh.warpMax[tid >> 5] = t;
  __syncthreads();
  if (tid == 0) {
    float m8 = -INFINITY;
    for (int i = 0; i < kThreads / 32; ++i)
      m8 = fmaxf(m8, sh.warpMax[i]);
    sh.thrTile = m8;
  }
  __syncthreads();
}

template <class Metric, class Weight>
__device__ __forceinline__ void nearestEpilogue(const Metric &m, const Weight &w,
                                                const PassState &sh, const ColumnMeta &cm,
                                                typename Metric::Acc (&acc)[8][8],
                                                const int (&rowComp)[8],
                                                const float (&rowVal)[8], int firstCol, int n,
                                                bool useComp, bool useValue, bool mask,
                                                const TileGeom &g, unsigned long long *rowBest) {
  float F[8];
  int cComp[8], cOrig[8];
  float cVal[8];
#pragma unroll
  for (int r = 0; r < 8; ++r)
    F[r] = sh.rowFilter[g.row(r)];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int col = g.col(c);
    const bool valid = firstCol + col < n;
    cOrig[c] = valid ? cm.orig[col] : -1;
    cComp[c] = valid ? (useComp ? cm.comp[col] : cOrig[c]) : -1;
    cVal[c] = useValue ? cm.value[col] : 0.0f;
  }
  // Fast path: does any pair of the warp pass its row's filter? Without
  // `mask` the minimum runs over every column, a superset of the pairs that
  // count, so it can only send more warps to the exact path below; `mask`
  // (tiles that may hold same-component pairs) excludes them up front.
  bool any = false;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    float mn = INFINITY;
    if (mask) {
#pragma unroll
      for (int c = 0; c < 8; ++c)
        mn = fminf(mn, cComp[c] != rowComp[r] ? m.filter(acc[r][c]) : INFINITY);
    } else {
#pragma unroll
      for (int c = 0; c < 8; ++c)
        mn = fminf(mn, m.filter(acc[r][c]));
    }
    any |= mn <= F[r];
  }
  if (!__any_sync(0xffffffffu, any))
    return;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    unsigned long long best = kEmptyKey;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const bool ok = cOrig[c] >= 0 && cComp[c] != rowComp[r] && m.filter(acc[r][c]) <= F[r];
      if (ok) {
        const float weight = w.weight(m.finalize(acc[r][c]), rowVal[r], cVal[c]);
        if (weight < INFINITY) {
          const unsigned long long key = packKey(weight, (uint32_t)cOrig[c]);
          best = key < best ? key : best;
        }
      }
    }
#pragma unroll
    for (int off = 8; off > 0; off /= 2) {
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, off);
      best = other < best ? other : best;
    }
    if (g.tc == 0 && best < rowBest[g.row(r)])
      rowBest[g.row(r)] = best;
  }
}

// Inserts value v of position j into a row's sorted k-NN list (v below the
// k-th value, which leaves the list); pos (the entries' positions) may be
// null.
// Walks down from the end four entries at a time (four independent loads per
// step): after the first tiles of a search most values that still enter a
// list land near its end, where this stops after one or two steps. The
// value goes after every entry <= v.
__device__ __forceinline__ void insertSortedPos(float *list, int *pos, int k, float v, int j) {
  int i = k - 1; // the slot being filled; list[k - 1] > v leaves the list
  for (; i >= 4; i -= 4) {
    const float a = list[i - 1], b = list[i - 2], c = list[i - 3], d = list[i - 4];
    int pa = 0, pb = 0, pc = 0, pd = 0;
    if (pos) {
      pa = pos[i - 1];
      pb = pos[i - 2];
      pc = pos[i - 3];
      pd = pos[i - 4];
    }
    if (!(a > v))
      goto place;
    list[i] = a;
    if (pos)
      pos[i] = pa;
    if (!(b > v)) {
      i -= 1;
      goto place;
    }
    list[i - 1] = b;
    if (pos)
      pos[i - 1] = pb;
    if (!(c > v)) {
      i -= 2;
      goto place;
    }
    list[i - 2] = c;
    if (pos)
      pos[i - 2] = pc;
    if (!(d > v)) {
      i -= 3;
      goto place;
    }
    list[i - 3] = d;
    if (pos)
      pos[i - 3] = pd;
  }
  for (; i > 0 && list[i - 1] > v; --i) {
    list[i] = list[i - 1];
    if (pos)
      pos[i] = pos[i - 1];
  }
place:
  list[i] = v;
  if (pos)
    pos[i] = j;
}

// Offers value v of position j to a row's k-NN list. Inserts it when it
// beats the k-th value and keeps `tie` = "some point outside the list lies at
// exactly the k-th value": an insertion evicts the old k-th, which ties the
// new k-th when they are equal (a smaller new k-th clears every earlier
// tie); a value equal to the k-th that stays out ties it. Returns whether v
// was inserted.
__device__ __forceinline__ bool knnOffer(float *list, int *pos, int k, float v, int j, int &tie) {
  const float kth = list[k - 1];
  if (v < kth) {
    insertSortedPos(list, pos, k, v, j);
    tie = (kth < INFINITY && list[k - 1] == kth) ? 1 : 0;
    return true;
  }
  if (v == kth)
    tie = 1;
  return false;
}

template <class Metric>
__device__ __forceinline__ void knnEpilogue(const Metric &m, PassState &sh, float *lists,
                                            int *listPos, int k,
                                            typename Metric::Acc (&acc)[8][8], int firstRow,
                                            int firstCol, int n, const int *colOrig,
                                            const TileGeom &g) {
  const int lane = threadIdx.x & 31;
  const unsigned groupMask = (lane < 16) ? 0x0000ffffu : 0xffff0000u;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int rowInTile = g.row(r);
    const int rowPos = firstRow + rowInTile;
    float *list = lists + rowInTile * k;
    const float F = sh.rowFilter[rowInTile];
    float mn = INFINITY;
#pragma unroll
    for (int c = 0; c < 8; ++c)
      mn = fminf(mn, m.filter(acc[r][c]));
    if (!__any_sync(0xffffffffu, rowPos < n && mn <= F))
      continue; // no pair of this row group can enter a list
    unsigned pending = 0;
    if (rowPos < n) {
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (firstCol + g.col(c) < n && colOrig[g.col(c)] >= 0 && m.filter(acc[r][c]) <= F)
          pending |= 1u << c;
    }
    while (true) {
      const unsigned lanes = __ballot_sync(0xffffffffu, pending != 0);
      if (lanes == 0)
        break;
      const unsigned group = lanes & groupMask;
      if (group != 0 && lane == __ffs(group) - 1) {
        const int c = __ffs(pending) - 1;
        pending &= pending - 1;
        typename Metric::Acc a = acc[r][0];
#pragma unroll
        for (int cc = 1; cc < 8; ++cc)
          if (cc == c)
            a = acc[r][cc];
        const int colPos = firstCol + g.col(c);
        // The point itself counts as distance 0 (hdbscan.cuh:205-212).
        const float v = colPos == rowPos ? 0.0f : fmaxf(m.finalize(a), 0.0f);
        knnOffer(list, listPos ? listPos + rowInTile * k : nullptr, k, v, colPos,
                 sh.rowTie[rowInTile]);
      }
      __syncwarp();
    }
  }
}

// Warp 0: collects candidate column tiles into sh.listTile / listLb, until the
// frontier is empty or the list is nearly full. Nodes whose bound exceeds the
// block threshold are dropped; subtrees of the row tile's own single
// component are skipped.
template <class Metric, class Weight>
__device__ void collectCandidates(const PassParams &p, const Metric &m, const Weight &w,
                                  PassState &sh, const float *rowLow, const float *rowHigh,
                                  int rowTile, int rowPure, float rowMinValue, float slack) {
  constexpr int kWidth = 2; // nodes per lane per step of the walk
  const int lane = threadIdx.x & 31;
  const float thr = sh.thrTile;
  int listLen = 0;
  int frontLen = sh.frontLen;
  while (frontLen > 0 && listLen <= kListCap - 32 * kWidth) {
    const int take = min(32 * kWidth, min(frontLen, kFrontierCap - frontLen));
    if (take == 0) {
      if (lane == 0)
        sh.overflow = 1;
      break;
    }
    int node[kWidth];
#pragma unroll
    for (int h = 0; h < kWidth; ++h)
      node[h] = lane + 32 * h < take ? sh.frontNode[frontLen - 1 - lane - 32 * h] : -1;
    __syncwarp();
    frontLen -= take;
    // Every field of every node of the step is loaded before any is used:
    // one round trip to L2 per step of the walk.
    int pure[kWidth], left[kWidth], right[kWidth], first[kWidth];
    float value[kWidth];
    typename Metric::Acc acc[kWidth];
#pragma unroll
    for (int h = 0; h < kWidth; ++h) {
      const int q = max(node[h], 0);
      pure[h] = p.nodePure ? __ldg(p.nodePure + q) : -1;
      left[h] = __ldg(p.nodeLeft + q);
      right[h] = __ldg(p.nodeRight + q);
      first[h] = __ldg(p.nodeFirstTile + q);
      value[h] = p.nodeMinValue ? __ldg(p.nodeMinValue + q) : 0.0f;
      acc[h] = m.init();
    }
    const bool box = p.prune && Metric::kBoxBound;
    if (box) {
#pragma unroll 4
      for (int f = 0; f < p.d; ++f) {
        const float rl = rowLow[f], rh = rowHigh[f];
#pragma unroll
        for (int h = 0; h < kWidth; ++h) {
          const size_t at = (size_t)max(node[h], 0) * p.d + f;
          const float gap = fmaxf(0.0f, fmaxf(__ldg(p.nodeLow + at) - rh, rl - __ldg(p.nodeHigh + at)));
          acc[h] = m.accumulate(acc[h], gap, 0.0f);
        }
      }
    }
#pragma unroll
    for (int h = 0; h < kWidth; ++h) {
      bool keepLeaf = false, expand = false;
      int tile = -1;
      float lb = 0.0f;
      if (node[h] >= 0) {
        const bool skip = rowPure >= 0 && pure[h] == rowPure;
        if (!skip && box)
          lb = w.lowerBound(m.finalize(acc[h]), rowMinValue, value[h]) * slack;
        if (!skip && lb <= thr) {
          if (left[h] < 0) {
            tile = first[h];
            keepLeaf = tile != rowTile;
            if (pure[h] >= 0)
              tile |= kPureColumnTile;
          } else {
            expand = true;
          }
        }
      }
      const unsigned leaves = __ballot_sync(0xffffffffu, keepLeaf);
      const unsigned inner = __ballot_sync(0xffffffffu, expand);
      const unsigned below = (1u << lane) - 1;
      if (keepLeaf) {
        const int at = listLen + __popc(leaves & below);
        sh.listTile[at] = tile;
        sh.listLb[at] = lb;
      }
      if (expand) {
        const int at = frontLen + 2 * __popc(inner & below);
        sh.frontNode[at] = left[h];
        sh.frontNode[at + 1] = right[h];
      }
      listLen += __popc(leaves);
      frontLen += 2 * __popc(inner);
    }
    __syncwarp();
  }
  if (lane == 0) {
    sh.listLen = listLen;
    sh.frontLen = frontLen;
  }
}

// Sorts the first `len` candidates by lower bound (bitonic network over the
// next power of two, padding with +inf). All threads call it.
__device__ __forceinline__ void sortCandidates(PassState &sh, int len) {
  int size = 1;
  while (size < len)
    size *= 2;
  for (int i = len + threadIdx.x; i < size; i += kThreads) {
    sh.listLb[i] = INFINITY;
    sh.listTile[i] = -1;
  }
  __syncthreads();
  for (int k = 2; k <= size; k *= 2) {
    for (int j = k / 2; j > 0; j /= 2) {
      for (int i = threadIdx.x; i < size / 2; i += kThreads) {
        const int lo = 2 * j * (i / j) + (i % j), hi = lo + j;
        const bool ascending = (lo & k) == 0;
        const float a = sh.listLb[lo], b = sh.listLb[hi];
        if ((a > b) == ascending) {
          sh.listLb[lo] = b;
          sh.listLb[hi] = a;
          const int t = sh.listTile[lo];
          sh.listTile[lo] = sh.listTile[hi];
          sh.listTile[hi] = t;
        }
      }
      __syncthreads();
    }
  }
}

template <class Metric, class Weight, int KC, bool kKnn>
__global__ void __launch_bounds__(kThreads, 2) passKernel(PassParams p, Metric m, Weight w) {
  extern __shared__ __align__(128) float dyn[];
  __shared__ PassState sh;
  // Dynamic layout: row tile, two column-tile buffers, two metadata buffers,
  // row box, k-NN lists. Every bulk-copy destination is 512-byte aligned.
  float *sA = dyn;
  float *sB[2] = {sA + KC * kTile, sA + 2 * KC * kTile};
  int *metaBase = (int *)(sA + 3 * KC * kTile);
  ColumnMeta meta[2];
  for (int b = 0; b < 2; ++b) {
    meta[b].orig = metaBase + b * 3 * kTile;
    meta[b].comp = metaBase + b * 3 * kTile + kTile;
    meta[b].value = (float *)(metaBase + b * 3 * kTile + 2 * kTile);
  }
  float *rowLow = (float *)(metaBase + 6 * kTile);
  float *rowHigh = rowLow + p.d;
  float *lists = rowHigh + p.d;
  int *listPos = (kKnn && p.knnPos) ? reinterpret_cast<int *>(lists + kTile * p.k) : nullptr;

  const TileGeom g;
  const int tid = threadIdx.x;
  const int I = p.tileOrder ? p.tileOrder[blockIdx.x] : (int)blockIdx.x;
  const int firstRow = I * kTile;
  const int leaf = p.leafOfTile[I];
  const int rowPure = (!kKnn && p.nodePure) ? p.nodePure[leaf] : -1;
  const float rowMinValue = p.nodeMinValue ? p.nodeMinValue[leaf] : 0.0f;
  const float slack = 1.0f - boxSlack(p.d);
  const bool useComp = !kKnn && p.component != nullptr;
  const bool useValue = !kKnn && w.value != nullptr;
  const size_t tileFloats = (size_t)p.numChunks * KC * kTile;

  int rowComp[8];
  float rowVal[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int pos = firstRow + g.row(r);
    const bool valid = pos < p.n;
    rowComp[r] = valid ? (p.component ? p.component[pos] : p.order[pos]) : -2;
    rowVal[r] = valid ? w.load(pos) : 0.0f;
  }
  if (tid < kTile) {
    const int pos = firstRow + tid;
    const unsigned long long seed =
        (!kKnn && p.seedKey && pos < p.n) ? p.seedKey[pos] : kEmptyKey;
    // A settled row keeps its seed as the answer (written before the pass).
    sh.rowBest[tid] = (seed & kSettledKey) && seed != kEmptyKey ? kEmptyKey : seed;
    sh.rowTie[tid] = 0;
  }
  if (kKnn)
    for (int i = tid; i < kTile * p.k; i += kThreads) {
      lists[i] = INFINITY;
      if (listPos)
        listPos[i] = -1;
    }
  for (int f = tid; f < p.d; f += kThreads) {
    rowLow[f] = p.nodeLow[(size_t)leaf * p.d + f];
    rowHigh[f] = p.nodeHigh[(size_t)leaf * p.d + f];
  }
  if (p.numChunks == 1)
    copyChunk(sA, p.tiled + (size_t)I * tileFloats, KC * kTile);
  if (tid == 0) {
    mbarrierInit(&sh.bar[0], 1);
    mbarrierInit(&sh.bar[1], 1);
    fenceBarrierInit();
    sh.frontLen = 0;
    sh.overflow = 0;
    const int root = p.rootOfTile ? p.rootOfTile[I] : 0;
    const int rootPure = (!kKnn && p.nodePure) ? p.nodePure[root] : -1;
    if (!(rowPure >= 0 && rootPure == rowPure)) {
      sh.frontNode[0] = root;
      sh.frontLen = 1;
    }
  }
  // Column metadata of the row tile itself, for the self tile.
  if (tid < kTile) {
    const int pos = firstRow + tid;
    const bool valid = pos < p.n;
    meta[0].orig[tid] = valid ? p.order[pos] : -1;
    if (useComp)
      meta[0].comp[tid] = valid ? p.component[pos] : -1;
    if (useValue)
      meta[0].value[tid] = valid ? w.load(pos) : 0.0f;
  }
  __syncthreads();
  refreshThresholds<Metric, Weight, kKnn>(p, m, w, sh, lists, firstRow);

  unsigned long long computed = 0;
  bool failed = false;

  // Accumulate + epilogue of one staged column tile.
  // Masking is needed only where same-component pairs can occur: not in
  // passes where every point is its own component, not between two tiles
  // that each hold a single (different) component.
  const bool maskPass = useComp && !p.singletons;
  auto processTile = [&](int J, const float *bTile, const ColumnMeta &cm, bool colPure) {
    typename Metric::Acc acc[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int c = 0; c < 8; ++c)
        acc[r][c] = m.init();
    accumulateChunk<Metric, KC>(sA, bTile, m, acc, g);
    if (kKnn)
      knnEpilogue(m, sh, lists, listPos, p.k, acc, firstRow, J * kTile, p.n, cm.orig, g);
    else
      nearestEpilogue<Metric, Weight>(m, w, sh, cm, acc, rowComp, rowVal, J * kTile, p.n,
                                      useComp, useValue,
                                      maskPass && !(rowPure >= 0 && colPure), g, sh.rowBest);
    __syncthreads();
    refreshThresholds<Metric, Weight, kKnn>(p, m, w, sh, lists, firstRow);
    ++computed;
  };
  // The general path (features in several chunks): synchronous staging.
  auto processTileChunked = [&](int J) {
    if (tid < kTile) {
      const int pos = J * kTile + tid;
      const bool valid = pos < p.n;
      meta[0].orig[tid] = valid ? p.order[pos] : -1;
      if (useComp)
        meta[0].comp[tid] = valid ? p.component[pos] : -1;
      if (useValue)
        meta[0].value[tid] = valid ? w.load(pos) : 0.0f;
    }
    typename Metric::Acc acc[8][8];
    computeTile<Metric, KC>(p.tiled, p.tiled, p.numChunks, I, J, sA, sB[0], m, acc, g);
    if (kKnn)
      knnEpilogue(m, sh, lists, listPos, p.k, acc, firstRow, J * kTile, p.n, meta[0].orig, g);
    else
      nearestEpilogue<Metric, Weight>(m, w, sh, meta[0], acc, rowComp, rowVal, J * kTile, p.n,
                                      useComp, useValue, maskPass, g, sh.rowBest);
    __syncthreads();
    refreshThresholds<Metric, Weight, kKnn>(p, m, w, sh, lists, firstRow);
    ++computed;
  };

  // 1. The row tile against itself (none if all its points share one
  //    component: no edge inside).
  if (rowPure < 0) {
    if (p.numChunks == 1)
      processTile(I, sA, meta[0], false);
    else
      processTileChunked(I);
  }

  // Issues the bulk copies of candidate `i` into buffer b (thread 0).
  const uint32_t metaBytes = (uint32_t)(kTile * sizeof(int)) * (1 + useComp + useValue);
  const uint32_t tileBytes = (uint32_t)(KC * kTile * sizeof(float));
  auto issue = [&](int i, int b) {
    const int J = sh.listTile[i] & ~kPureColumnTile;
    fenceProxyAsync();
    mbarrierArriveExpectTx(&sh.bar[b], tileBytes + metaBytes);
    bulkCopyToShared(sB[b], p.tiled + (size_t)J * tileFloats, tileBytes, &sh.bar[b]);
    bulkCopyToShared(meta[b].orig, p.order + (size_t)J * kTile, kTile * sizeof(int), &sh.bar[b]);
    if (useComp)
      bulkCopyToShared(meta[b].comp, p.component + (size_t)J * kTile, kTile * sizeof(int),
                       &sh.bar[b]);
    if (useValue)
      bulkCopyToShared(meta[b].value, w.value + (size_t)J * kTile, kTile * sizeof(float),
                       &sh.bar[b]);
  };
  uint32_t phase[2] = {0, 0};
  bool inFlight[2] = {false, false};

  while (!failed) {
    // 2. Candidates of this batch.
    if (tid < 32)
      collectCandidates(p, m, w, sh, rowLow, rowHigh, I, rowPure, rowMinValue, slack);
    __syncthreads();
    const int len = sh.listLen;
    if (sh.overflow) {
      failed = true;
      break;
    }
    if (len == 0 && sh.frontLen == 0)
      break;
    // 3. Nearest first.
    if (p.prune && Metric::kBoxBound && len > 1)
      sortCandidates(sh, len);
    // 4. Compute them.
    if (p.numChunks == 1) {
      auto nextValid = [&](int from) {
        while (from < len && sh.listLb[from] > sh.thrTile)
          ++from;
        return from;
      };
      int cur = nextValid(0), buf = 0;
      if (cur < len) {
        if (tid == 0)
          issue(cur, buf);
        inFlight[buf] = true;
      }
      while (cur < len) {
        const int next = nextValid(cur + 1);
        if (next < len) {
          if (tid == 0)
            issue(next, buf ^ 1);
          inFlight[buf ^ 1] = true;
        }
        const bool ready = mbarrierWait(&sh.bar[buf], phase[buf]);
        phase[buf] ^= 1;
        inFlight[buf] = false;
        if (__syncthreads_or(!ready)) {
          failed = true;
          break;
        }
        if (sh.listLb[cur] <= sh.thrTile)
          processTile(sh.listTile[cur] & ~kPureColumnTile, sB[buf], meta[buf],
                      (sh.listTile[cur] & kPureColumnTile) != 0);
        else
          __syncthreads(); // nobody reads this buffer any more
        cur = next;
        buf ^= 1;
      }
    } else {
      for (int i = 0; i < len; ++i)
        if (sh.listLb[i] <= sh.thrTile)
          processTileChunked(sh.listTile[i] & ~kPureColumnTile);
    }
    __syncthreads();
    if (sh.frontLen == 0)
      break;
  }

  // After a failed wait, give copies still in flight a bounded chance to land
  // before the block's shared memory is released.
  for (int b = 0; b < 2; ++b)
    if (inFlight[b])
      mbarrierWait(&sh.bar[b], phase[b]);
  if (tid < kTile) {
    const int pos = firstRow + tid;
    if (pos < p.n) {
      if (kKnn) {
        const int rank = p.coreRank ? p.coreRank[pos] : p.k;
        p.core[pos] = rank > 0 ? lists[tid * p.k + rank - 1] : 0.0f;
        if (listPos) {
          for (int e = 0; e < p.k; ++e)
            p.knnPos[(size_t)pos * p.k + e] = listPos[tid * p.k + e];
          p.knnTie[pos] = sh.rowTie[tid];
        }
      } else if ((!p.radius || p.radius[pos] >= 0.0f) &&
                 !(p.seedKey && (p.seedKey[pos] & kSettledKey) &&
                   p.seedKey[pos] != kEmptyKey)) {
        p.nearest[pos] = sh.rowBest[tid];
      }
    }
  }
  if (tid == 0) {
    if (p.tileWork)
      p.tileWork[I] = (unsigned int)computed;
    if (p.tilesComputed)
      atomicAdd(p.tilesComputed, computed);
    if (failed && p.error)
      atomicCAS(p.error, 0, sh.overflow ? (int)kErrorTooLarge : (int)kErrorTimeout);
  }
}

// Host launcher. KC follows the point layout (chunkWidthFor(d)).
template <class Metric, class Weight, bool kKnn>
int launchPass(const PassParams &p, const Metric &m, const Weight &w, int kc,
               cudaStream_t stream) {
  const size_t listEntries = kKnn ? (size_t)kTile * p.k * (p.knnPos ? 2 : 1) : 0;
  const size_t dynBytes = (size_t)3 * kc * kTile * sizeof(float) + 6 * kTile * sizeof(int) +
                          (2 * (size_t)p.d + listEntries) * sizeof(float);
  // Bulk copies need 16-byte aligned sources (pool allocations are 256-byte
  // aligned; refuse anything else rather than fault).
  auto misaligned = [](const void *ptr) { return ((uintptr_t)ptr & 15) != 0; };
  if (misaligned(p.tiled) || misaligned(p.order) || misaligned(p.component) ||
      misaligned(w.value))
    return (int)cudaErrorMisalignedAddress;
  auto run = [&](auto kernel) {
    // Static (~18 KB) plus dynamic shared memory can pass the 48 KB default.
    const cudaError_t e =
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dynBytes);
    if (e != cudaSuccess)
      return (int)e;
    kernel<<<p.numTiles, kThreads, dynBytes, stream>>>(p, m, w);
    noteLaunch();
    return (int)cudaGetLastError();
  };
  switch (kc) {
  case 4:
    return run(passKernel<Metric, Weight, 4, kKnn>);
  case 8:
    return run(passKernel<Metric, Weight, 8, kKnn>);
  case 16:
    return run(passKernel<Metric, Weight, 16, kKnn>);
  default:
    return run(passKernel<Metric, Weight, 32, kKnn>);
  }
}

} // namespace cuhc
