// Borůvka rounds on the GPU (template bodies; instantiated per metric).
//
// Round structure (the reference runs steps 2-5 on the CPU with two
// synchronous copies per round, mst.cuh:118-181; here nothing leaves the
// device but two counters):
//   1. BVH purity of the current components; each component's best known
//      edge weight is seeded from last round's per-point edges that now
//      leave it (a valid upper bound that lets the pass prune at once);
//   2. the pass: per point, its minimum edge to another component;
//   3. per component, the minimum edge under the order (weight, u, v) with
//      ORIGINAL indices: an atomicMin over (weight bits << 32 | u), then an
//      atomicMin over v among the points that hold that (weight, u). Any
//      point's best edge ties toward the lower other endpoint, which is also
//      the lower edge under (u, v) for that point, so the component minimum
//      is the minimum over its points (as in the reference's CPU loop);
//   4. hooking: each component points at the component across its edge; a
//      pair that chose the same edge keeps the lower label as root and adds
//      the edge once. With one strict total order on edges the chosen edges
//      form a forest plus those 2-cycles, so this is cycle free;
//   5. pointer jumping to the roots, relabel, count components and edges.
#pragma once

#include <algorithm>

#include "profiling.cuh"
#include "mst.cuh"
#include "passes.cuh"
#include "screen.cuh"

namespace cuhc {
namespace boruvka_detail {

inline int blocks(long long work, int threads = 256) { return (int)((work + threads - 1) / threads); }

static __global__ void iotaKernel(int *a, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    a[i] = i;
}

static __global__ void fillU32(unsigned int *a, unsigned int v, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    a[i] = v;
}

// compBest[comp[i]] <- min over i of last round's edge weights that leave
// the (new) component of i.
static __global__ void seedComponentBest(const unsigned long long *__restrict__ nearest,
                                  const int *__restrict__ rank, const int *__restrict__ comp,
                                  unsigned int *__restrict__ compBest, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const unsigned long long key = nearest[i];
  if (key == kEmptyKey)
    return;
  const int j = rank[keyIndex(key)];
  if (comp[j] != comp[i])
    atomicMin(&compBest[comp[i]], (unsigned int)(key >> 32));
}

static __global__ void componentKeyPass1(const unsigned long long *__restrict__ nearest,
                                  const int *__restrict__ order, const int *__restrict__ comp,
                                  unsigned long long *__restrict__ compKey, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const unsigned long long key = nearest[i];
  if (key == kEmptyKey)
    return;
  const uint32_t oi = (uint32_t)order[i], oj = keyIndex(key);
  const unsigned long long k1 = (key & 0xffffffff00000000ull) | (oi < oj ? oi : oj);
  atomicMin(&compKey[comp[i]], k1);
}

static __global__ void componentKeyPass2(const unsigned long long *__restrict__ nearest,
                                  const int *__restrict__ order, const int *__restrict__ comp,
                                  const unsigned long long *__restrict__ compKey,
                                  unsigned int *__restrict__ compV, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  const unsigned long long key = nearest[i];
  if (key == kEmptyKey)
    return;
  const uint32_t oi = (uint32_t)order[i], oj = keyIndex(key);
  const unsigned long long k1 = (key & 0xffffffff00000000ull) | (oi < oj ? oi : oj);
  if (k1 == compKey[comp[i]])
    atomicMin(&compV[comp[i]], oi < oj ? oj : oi);
}

// One thread per position that is a component root (comp[r] == r).
static __global__ void hookComponents(const int *__restrict__ comp, const int *__restrict__ rank,
                               const unsigned long long *__restrict__ compKey,
                               const unsigned int *__restrict__ compV, int *__restrict__ parent,
                               int *__restrict__ edgeU, int *__restrict__ edgeV,
                               float *__restrict__ edgeW, int *__restrict__ counters,
                               int edgeCapacity, int n) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n || comp[r] != r)
    return;
  const unsigned long long k1 = compKey[r];
  if (k1 == kEmptyKey) {
    parent[r] = r;
    return;
  }
  const int u = (int)keyIndex(k1), v = (int)compV[r];
  const int cu = comp[rank[u]], cv = comp[rank[v]];
  const int t = cu == r ? cv : cu;
  const bool mutual = compKey[t] == k1 && compV[t] == (unsigned int)v;
  bool add = true;
  if (mutual && r > t) {
    add = false; // the lower label adds the shared edge
  }
  parent[r] = (mutual && r < t) ? r : t;
  if (add) {
    const int slot = atomicAdd(&counters[0], 1);
    if (slot >= edgeCapacity)
      return; // more edges than a tree has: the host reports the error
    edgeU[slot] = u;
    edgeV[slot] = v;
    edgeW[slot] = keyWeight(k1);
  }
}

static __global__ void jumpParents(const int *__restrict__ comp, int *__restrict__ parent, int n) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n || comp[r] != r)
    return;
  parent[r] = parent[parent[r]];
}

static __global__ void countRoots(const int *__restrict__ comp, const int *__restrict__ parent,
                           int *__restrict__ counters, int n) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n || comp[r] != r)
    return;
  if (parent[r] == r)
    atomicAdd(&counters[1], 1);
  if (parent[parent[r]] != parent[r])
    atomicAdd(&counters[2], 1); // not fully jumped (would be a bug)
}

static __global__ void relabel(int *__restrict__ comp, const int *__restrict__ parent, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    comp[i] = parent[comp[i]];
}

} // namespace boruvka_detail

template <class Metric, class Weight>
int boruvkaMst(SpatialIndex &index, const Metric &metric, const Weight &weight, bool prune,
               DeviceEdges &edges, PassStats *stats, cudaStream_t stream) {
  using namespace boruvka_detail;
  const int n = index.n;
  StatusChain st;
  edges.count = 0;
  CUHC_TRY(st, edges.u.allocate(std::max(n - 1, 1), stream));
  CUHC_TRY(st, edges.v.allocate(std::max(n - 1, 1), stream));
  CUHC_TRY(st, edges.w.allocate(std::max(n - 1, 1), stream));
  if (n < 2 || !st.ok())
    return st.code;

  DeviceBuffer<int> comp, parent, counters, error;
  DeviceBuffer<unsigned long long> nearest, compKey, tiles;
  DeviceBuffer<unsigned int> compBest, compV;
  CUHC_TRY(st, comp.allocate(paddedToTiles(n), stream));
  CUHC_TRY(st, parent.allocate(n, stream));
  CUHC_TRY(st, counters.allocate(4, stream));
  CUHC_TRY(st, error.allocate(1, stream));
  CUHC_TRY(st, nearest.allocate(n, stream));
  CUHC_TRY(st, compKey.allocate(n, stream));
  CUHC_TRY(st, tiles.allocate(1, stream));
  CUHC_TRY(st, compBest.allocate(n, stream));
  CUHC_TRY(st, compV.allocate(n, stream));
  if (!st.ok())
    return st.code;
  iotaKernel<<<blocks(n), 256, 0, stream>>>(comp.get(), n); noteLaunch();
  CUHC_TRY(st, cudaMemsetAsync(nearest.get(), 0xff, n * sizeof(unsigned long long), stream));
  CUHC_TRY(st, cudaMemsetAsync(error.get(), 0, sizeof(int), stream));
  CUHC_TRY(st, cudaMemsetAsync(tiles.get(), 0, sizeof(unsigned long long), stream));

  PassParams p{};
  p.tiled = index.tiled.get();
  p.n = n;
  p.d = index.d;
  p.numChunks = index.numChunks;
  p.numTiles = index.numTiles;
  p.order = index.order.get();
  p.component = comp.get();
  p.nodeLeft = index.nodeLeft.get();
  p.nodeRight = index.nodeRight.get();
  p.nodeFirstTile = index.nodeFirstTile.get();
  p.leafOfTile = index.leafOfTile.get();
  p.nodePure = index.nodePure.get();
  p.nodeLow = index.nodeLow.get();
  p.nodeHigh = index.nodeHigh.get();
  p.nodeMinValue = index.hasMinValues ? index.nodeMinValue.get() : nullptr;
  p.prune = prune;
  p.nearest = nearest.get();
  p.compBest = compBest.get();
  p.tilesComputed = tiles.get();
  p.error = error.get();
  p.screenStats = screenCounters();

  const bool screened = useScreen<Metric>(index.d, 0) && index.extentsWithin(kScreenMaxExtent);
  int numComponents = n, totalEdges = 0, rounds = 0;
  unsigned long long tilesSoFar = 0;
  int hostCounters[4];
  while (st.ok() && numComponents > 1) {
    CUHC_TRY(st, index.updatePurity(comp.get()));
    fillU32<<<blocks(n), 256, 0, stream>>>(compBest.get(), 0x7f800000u, n); noteLaunch();
    if (rounds > 0) {
      seedComponentBest<<<blocks(n), 256, 0, stream>>>(nearest.get(), index.rank.get(),
                                                       comp.get(), compBest.get(), n);
      noteLaunch();
    }
    CUHC_TRY(st, cudaGetLastError());
    p.singletons = rounds == 0;
    {
      PassTimer timer(screened ? kTimerScreenPass : kTimerNearestPass, stream);
      if (screened)
        CUHC_TRY(st, (launchScreen<Metric, Weight, false>(p, metric, weight, index.kc, stream)));
      else
        CUHC_TRY(st, (launchPass<Metric, Weight, false>(p, metric, weight, index.kc, stream)));
      if (timer.start) {
        unsigned long long tilesNow = 0;
        cudaMemcpyAsync(&tilesNow, tiles.get(), sizeof(tilesNow), cudaMemcpyDeviceToHost, stream);
        timer.finish(tilesNow - tilesSoFar);
        tilesSoFar = tilesNow;
      }
    }
    CUHC_TRY(st, cudaMemsetAsync(compKey.get(), 0xff, n * sizeof(unsigned long long), stream));
    CUHC_TRY(st, cudaMemsetAsync(compV.get(), 0xff, n * sizeof(unsigned int), stream));
    CUHC_TRY(st, cudaMemsetAsync(counters.get(), 0, 4 * sizeof(int), stream));
    componentKeyPass1<<<blocks(n), 256, 0, stream>>>(nearest.get(), index.order.get(), comp.get(),
                                                     compKey.get(), n); noteLaunch();
    componentKeyPass2<<<blocks(n), 256, 0, stream>>>(nearest.get(), index.order.get(), comp.get(),
                                                     compKey.get(), compV.get(), n); noteLaunch();
    hookComponents<<<blocks(n), 256, 0, stream>>>(
        comp.get(), index.rank.get(), compKey.get(), compV.get(), parent.get(),
        edges.u.get() + totalEdges, edges.v.get() + totalEdges, edges.w.get() + totalEdges,
        counters.get(), n - 1 - totalEdges, n); noteLaunch();
    int jumps = 1;
    while ((1 << jumps) < numComponents)
      ++jumps;
    for (int j = 0; j <= jumps; ++j) {
      jumpParents<<<blocks(n), 256, 0, stream>>>(comp.get(), parent.get(), n);
      noteLaunch();
    }
    countRoots<<<blocks(n), 256, 0, stream>>>(comp.get(), parent.get(), counters.get(), n); noteLaunch();
    relabel<<<blocks(n), 256, 0, stream>>>(comp.get(), parent.get(), n); noteLaunch();
    CUHC_TRY(st, cudaGetLastError());
    int passError = 0;
    CUHC_TRY(st, cudaMemcpyAsync(hostCounters, counters.get(), 4 * sizeof(int),
                                 cudaMemcpyDeviceToHost, stream));
    CUHC_TRY(st, cudaMemcpyAsync(&passError, error.get(), sizeof(int), cudaMemcpyDeviceToHost,
                                 stream));
    CUHC_TRY(st, cudaStreamSynchronize(stream));
    if (!st.ok())
      break;
    ++rounds;
    if (passError != 0) {
      st(passError);
      break;
    }
    const int added = hostCounters[0];
    if (hostCounters[2] != 0) {
      st(kErrorTimeout);
      break;
    }
    if (added == 0) {
      st(kErrorDisconnected);
      break;
    }
    totalEdges += added;
    numComponents = hostCounters[1];
    if (totalEdges > n - 1) {
      st(kErrorNonFinite);
      break;
    }
  }
  int err = 0;
  unsigned long long tileCount = 0;
  CUHC_TRY(st, cudaMemcpyAsync(&err, error.get(), sizeof(int), cudaMemcpyDeviceToHost, stream));
  CUHC_TRY(st, cudaMemcpyAsync(&tileCount, tiles.get(), sizeof(tileCount),
                               cudaMemcpyDeviceToHost, stream));
  CUHC_TRY(st, cudaStreamSynchronize(stream));
  if (err)
    st(err);
  edges.count = totalEdges;
  if (stats) {
    stats->tilesComputed += tileCount;
    stats->tilesTotal += (unsigned long long)rounds * index.numTiles * index.numTiles;
    stats->passes += rounds;
    stats->rounds += rounds;
  }
  return st.code;
}

template <class Metric>
int coreDistances(SpatialIndex &index, const Metric &metric, int k, bool prune, float *core,
                  PassStats *stats, cudaStream_t stream) {
  StatusChain st;
  DeviceBuffer<unsigned long long> tiles;
  DeviceBuffer<int> error;
  CUHC_TRY(st, tiles.allocate(1, stream));
  CUHC_TRY(st, error.allocate(1, stream));
  CUHC_TRY(st, cudaMemsetAsync(tiles.get(), 0, sizeof(unsigned long long), stream));
  CUHC_TRY(st, cudaMemsetAsync(error.get(), 0, sizeof(int), stream));
  if (!st.ok())
    return st.code;
  PassParams p{};
  p.tiled = index.tiled.get();
  p.n = index.n;
  p.d = index.d;
  p.numChunks = index.numChunks;
  p.numTiles = index.numTiles;
  p.order = index.order.get();
  p.component = nullptr;
  p.nodeLeft = index.nodeLeft.get();
  p.nodeRight = index.nodeRight.get();
  p.nodeFirstTile = index.nodeFirstTile.get();
  p.leafOfTile = index.leafOfTile.get();
  p.nodePure = nullptr;
  p.nodeLow = index.nodeLow.get();
  p.nodeHigh = index.nodeHigh.get();
  p.nodeMinValue = nullptr;
  p.prune = prune;
  p.core = core;
  p.k = k;
  p.tilesComputed = tiles.get();
  p.error = error.get();
  p.screenStats = screenCounters();
  {
    const bool screened =
        useScreen<Metric>(index.d, k) && index.extentsWithin(kScreenMaxExtent);
    PassTimer timer(screened ? kTimerScreenKnnPass : kTimerKnnPass, stream);
    if (screened)
      CUHC_TRY(st, (launchScreen<Metric, PlainWeight, true>(p, metric, PlainWeight{}, index.kc,
                                                            stream)));
    else
      CUHC_TRY(st, (launchPass<Metric, PlainWeight, true>(p, metric, PlainWeight{}, index.kc,
                                                          stream)));
    if (timer.start) {
      unsigned long long tilesNow = 0;
      cudaMemcpyAsync(&tilesNow, tiles.get(), sizeof(tilesNow), cudaMemcpyDeviceToHost, stream);
      timer.finish(tilesNow);
    }
  }
  int err = 0;
  unsigned long long tileCount = 0;
  CUHC_TRY(st, cudaMemcpyAsync(&err, error.get(), sizeof(int), cudaMemcpyDeviceToHost, stream));
  CUHC_TRY(st, cudaMemcpyAsync(&tileCount, tiles.get(), sizeof(tileCount),
                               cudaMemcpyDeviceToHost, stream));
  CUHC_TRY(st, cudaStreamSynchronize(stream));
  if (err)
    st(err);
  if (stats) {
    stats->tilesComputed += tileCount;
    stats->tilesTotal += (unsigned long long)index.numTiles * index.numTiles;
    stats->passes += 1;
  }
  return st.code;
}

} // namespace cuhc
