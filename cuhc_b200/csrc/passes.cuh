// The two all-pairs pass kernels (see engine.cuh for the block shape):
//
//   nearestPassKernel  for every point, its minimum-weight edge to a point of
//                      another component, key (weight bits, original index);
//                      the Borůvka step (single linkage, HDBSCAN) and the
//                      RNN-Ward nearest-cluster step (every slot its own
//                      component). Same result as the reference's
//                      nearestOtherComponent{,Symmetric,Walk}Kernel
//                      (distance_matrix.cuh:228-390, spatial.cuh:215-343) for
//                      every row whose component can still win; rows of a
//                      component whose best edge is known to be lighter may
//                      stop early, which never changes the component minimum.
//   knnPassKernel      for every point, the k-th smallest distance with the
//                      point itself counted as 0 (HDBSCAN core distances);
//                      same values as the reference's kthNearestFusedKernel
//                      (hdbscan.cuh:144-258).
#pragma once

#include "profiling.cuh"
#include "engine.cuh"

namespace cuhc {

// Threads 0..127 (one row each) refresh the row filters and the tile
// threshold; everyone must call it (it synchronizes).
template <class Metric, class Weight, bool kKnn>
__device__ __forceinline__ void refreshThresholds(const PassParams &p, const Metric &m,
                                                  const Weight &w, PassShared &sh,
                                                  const float *lists, int firstRow) {
  const int tid = threadIdx.x;
  float t = -INFINITY;
  if (tid < kTile) {
    const int pos = firstRow + tid;
    const bool valid = pos < p.n;
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
      const float v = valid ? w.load(pos) : 0.0f;
      if (valid && w.feasible(thr, v))
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

// Column data of tile J into shared memory (threads 0..127).
template <class Weight>
__device__ __forceinline__ void loadColumns(const PassParams &p, const Weight &w, PassShared &sh,
                                            int tileJ) {
  const int tid = threadIdx.x;
  if (tid < kTile) {
    const int pos = tileJ * kTile + tid;
    const bool valid = pos < p.n;
    const int orig = valid ? p.order[pos] : -1;
    sh.colOrig[tid] = orig;
    sh.colComp[tid] = valid ? (p.component ? p.component[pos] : orig) : -1;
    sh.colValue[tid] = valid ? w.load(pos) : 0.0f;
  }
}

template <class Metric, class Weight, int KC>
__device__ __forceinline__ void nearestEpilogue(const Metric &m, const Weight &w, PassShared &sh,
                                                typename Metric::Acc (&acc)[8][8],
                                                const int (&rowComp)[8],
                                                const float (&rowVal)[8], const TileGeom &g) {
  float F[8];
  int cComp[8], cOrig[8];
  float cVal[8];
#pragma unroll
  for (int r = 0; r < 8; ++r)
    F[r] = sh.rowFilter[g.row(r)];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int col = g.col(c);
    cComp[c] = sh.colComp[col];
    cOrig[c] = sh.colOrig[col];
    cVal[c] = sh.colValue[col];
  }
  bool any = false;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    float mn = INFINITY;
    bool seen = false;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const bool ok = cOrig[c] >= 0 && cComp[c] != rowComp[r];
      mn = fminf(mn, ok ? m.filter(acc[r][c]) : INFINITY);
      seen |= ok;
    }
    any |= seen && mn <= F[r];
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
    if (g.tc == 0 && best < sh.rowBest[g.row(r)])
      sh.rowBest[g.row(r)] = best;
  }
}

__device__ __forceinline__ void insertSorted(float *list, int k, float v) {
  if (!(v < list[k - 1]))
    return;
  int pos = k - 1;
  while (pos > 0 && list[pos - 1] > v) {
    list[pos] = list[pos - 1];
    --pos;
  }
  list[pos] = v;
}

template <class Metric>
__device__ __forceinline__ void knnEpilogue(const Metric &m, PassShared &sh, float *lists, int k,
                                            typename Metric::Acc (&acc)[8][8], int firstRow,
                                            int firstCol, int n, const TileGeom &g) {
  const int lane = threadIdx.x & 31;
  const unsigned groupMask = (lane < 16) ? 0x0000ffffu : 0xffff0000u;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int rowInTile = g.row(r);
    const int rowPos = firstRow + rowInTile;
    float *list = lists + rowInTile * k;
    const float F = sh.rowFilter[rowInTile];
    unsigned pending = 0;
    if (rowPos < n) {
#pragma unroll
      for (int c = 0; c < 8; ++c)
        if (sh.colOrig[g.col(c)] >= 0 && m.filter(acc[r][c]) <= F)
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
        insertSorted(list, k, v);
      }
      __syncwarp();
    }
  }
}

template <class Metric, class Weight, int KC, bool kKnn>
__global__ void __launch_bounds__(kThreads, 2)
    passKernel(PassParams p, Metric m, Weight w) {
  extern __shared__ __align__(16) float dyn[];
  __shared__ PassShared sh;
  float *sA = dyn;
  float *sB = sA + KC * kTile;
  float *rowLow = sB + KC * kTile;
  float *rowHigh = rowLow + p.d;
  float *lists = rowHigh + p.d; // knn only: [128][k]

  const TileGeom g;
  const int tid = threadIdx.x;
  const int I = blockIdx.x;
  const int firstRow = I * kTile;
  const int leaf = p.leafOfTile[I];
  const int rowPure = (!kKnn && p.nodePure) ? p.nodePure[leaf] : -1;
  const float rowMinValue = p.nodeMinValue ? p.nodeMinValue[leaf] : 0.0f;
  const float slack = 1.0f - boxSlack(p.d);

  int rowComp[8];
  float rowVal[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int pos = firstRow + g.row(r);
    const bool valid = pos < p.n;
    rowComp[r] = valid ? (p.component ? p.component[pos] : p.order[pos]) : -2;
    rowVal[r] = valid ? w.load(pos) : 0.0f;
  }
  if (tid < kTile)
    sh.rowBest[tid] = kEmptyKey;
  if (kKnn)
    for (int i = tid; i < kTile * p.k; i += kThreads)
      lists[i] = INFINITY;
  for (int f = tid; f < p.d; f += kThreads) {
    rowLow[f] = p.nodeLow[(size_t)leaf * p.d + f];
    rowHigh[f] = p.nodeHigh[(size_t)leaf * p.d + f];
  }
  if (p.numChunks == 1)
    copyChunk(sA, p.tiled + (size_t)I * KC * kTile, KC * kTile);
  if (tid == 0) {
    sh.sp = 0;
    sh.overflow = 0;
    const int root = 0;
    const int rootPure = p.nodePure && !kKnn ? p.nodePure[root] : -1;
    if (!(rowPure >= 0 && rootPure == rowPure)) {
      sh.stackNode[0] = root;
      sh.stackLb[0] = 0.0f;
      sh.sp = 1;
    }
  }
  __syncthreads();
  refreshThresholds<Metric, Weight, kKnn>(p, m, w, sh, lists, firstRow);

  unsigned long long computed = 0;
  // The row tile against itself first: it seeds every threshold with the
  // nearest points in space. A tile whose points share one component has no
  // edge inside.
  int J = rowPure >= 0 ? -1 : I;
  while (true) {
    if (J >= 0) {
      loadColumns(p, w, sh, J);
      typename Metric::Acc acc[8][8];
      computeTile<Metric, KC>(p.tiled, p.tiled, p.numChunks, I, J, sA, sB, m, acc, g);
      if (kKnn)
        knnEpilogue(m, sh, lists, p.k, acc, firstRow, J * kTile, p.n, g);
      else
        nearestEpilogue<Metric, Weight, KC>(m, w, sh, acc, rowComp, rowVal, g);
      __syncthreads();
      refreshThresholds<Metric, Weight, kKnn>(p, m, w, sh, lists, firstRow);
      ++computed;
    }
    if (tid < 32)
      traverseNext(p, m, w, sh, rowLow, rowHigh, I, rowPure, rowMinValue, slack);
    __syncthreads();
    J = sh.next;
    if (J < 0)
      break;
  }

  if (tid < kTile) {
    const int pos = firstRow + tid;
    if (pos < p.n) {
      if (kKnn)
        p.core[pos] = lists[tid * p.k + p.k - 1];
      else
        p.nearest[pos] = sh.rowBest[tid];
    }
  }
  if (tid == 0) {
    if (p.tilesComputed)
      atomicAdd(p.tilesComputed, computed);
    if (sh.overflow && p.error)
      atomicCAS(p.error, 0, (int)kErrorTooLarge);
  }
}

// Host launcher. KC follows the point layout (chunkWidthFor(d)).
template <class Metric, class Weight, bool kKnn>
int launchPass(const PassParams &p, const Metric &m, const Weight &w, int kc,
               cudaStream_t stream) {
  const size_t dynBytes =
      (size_t)(2 * kc * kTile + 2 * p.d + (kKnn ? kTile * p.k : 0)) * sizeof(float);
  auto run = [&](auto kernel) {
    if (dynBytes > 48 * 1024) {
      const cudaError_t e =
          cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dynBytes);
      if (e != cudaSuccess)
        return (int)e;
    }
    kernel<<<p.numTiles, kThreads, dynBytes, stream>>>(p, m, w); noteLaunch();
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
