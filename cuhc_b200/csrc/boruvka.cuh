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
#include <typeinfo>
#include <tuple>
#include <mutex>
#include <map>
#include <random>
#include <type_traits>

#include "profiling.cuh"
#include "mst.cuh"
#include "passes.cuh"
#include "screen.cuh"

namespace cuhc {
// Sets the calling thread's screened pipeline shape for a scope.
struct ScreenShapeScope {
  ScreenShape previous;
  explicit ScreenShapeScope(ScreenShape shape) : previous(currentScreenShape()) {
    setScreenShape(shape);
  }
  ~ScreenShapeScope() { setScreenShape(previous); }
};

// Pipeline-shape tuner of the screened k-NN pass (defined below).
template <class Metric>
ScreenShape tunedScreenShape(SpatialIndex &index, const Metric &m, int k, float *scratch,
                             cudaStream_t s);

// Whether the index's data suits the metric's tensor-core screen (callers
// check useScreen too): coordinate extents for every screened metric, and for
// cosine the range of the points' squared norms.
template <class Metric> inline bool screenDataOk(SpatialIndex &index) {
  if (!index.extentsWithin(kScreenMaxExtent))
    return false;
  if constexpr (std::is_same<Metric, CosineMetric>::value)
    return index.normsWithin(kCosineNormLow, kCosineNormHigh);
  return true;
}

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

// The screened pass's per-tile metadata of a round: [orig, comp, value] x
// 128 slots per tile (PassParams::packedMeta); slots past n hold -1, 0, 0.
static __global__ void packMeta(const int *__restrict__ order, const int *__restrict__ comp,
                                const float *__restrict__ value, int n, int numTiles,
                                int *__restrict__ packed) {
  const int pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= numTiles * kTile)
    return;
  int *tile = packed + (size_t)(pos / kTile) * 3 * kTile + pos % kTile;
  const bool real = pos < n;
  tile[0] = real ? order[pos] : -1;
  tile[kTile] = real ? comp[pos] : 0;
  tile[2 * kTile] = real && value ? __float_as_int(value[pos]) : 0;
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

// Seeds of a round from HDBSCAN's k-NN lists (mutual reachability, alpha
// 1). A list member j of row i lies within core_i, so the edge (i, j) weighs
// max(core_i, core_j) (fmaxf is exact: the pass computes the same bits).
// Per row: seed = the lightest such edge to another component, under the
// key order (weight, original index), and its weight goes into the
// component's best (a real edge: a valid bound). The seed is the row's final
// answer when it weighs core_i and no point outside the list ties the k-th
// distance: every point outside the list is then farther than core_i, so its
// edge weighs more than core_i, the least any edge of row i can weigh. Such a
// row is settled: its answer goes to nearest now and the pass skips it.
static __global__ void seedFromKnn(const int *__restrict__ knnPos, const int *__restrict__ knnTie,
                                   int k, const float *__restrict__ core,
                                   const int *__restrict__ order, const int *__restrict__ comp,
                                   unsigned long long *__restrict__ seed,
                                   unsigned long long *__restrict__ nearest,
                                   unsigned int *__restrict__ compBest, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  if (order[i] < 0) {
    seed[i] = kEmptyKey;
    return;
  }
  const float ci = core[i];
  const int c = comp[i];
  unsigned long long best = kEmptyKey;
  const int *list = knnPos + (size_t)i * k;
  for (int e = 0; e < k; ++e) {
    const int j = list[e];
    if (j < 0 || j == i || comp[j] == c)
      continue;
    const unsigned long long key = packKey(fmaxf(ci, core[j]), (uint32_t)order[j]);
    best = key < best ? key : best;
  }
  if (best == kEmptyKey) {
    seed[i] = kEmptyKey;
    return;
  }
  atomicMin(&compBest[c], (unsigned int)(best >> 32));
  const bool settled = keyWeight(best) == ci && knnTie[i] == 0;
  seed[i] = settled ? (best | kSettledKey) : best;
  if (settled)
    nearest[i] = best;
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
               DeviceEdges &edges, PassStats *stats, cudaStream_t stream, RadiusLog *radiusLog,
               const KnnLists *knn) {
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
  p.screenAudit = screenAuditWords();
  p.rootOfTile = index.numInstances > 1 ? index.rootOfTile.get() : nullptr;

  const bool screened = useScreen<Metric>(index.d, 0) && screenDataOk<Metric>(index);
  DeviceBuffer<int> packed;
  if (screened)
    CUHC_TRY(st, packed.allocate((size_t)index.numTiles * 3 * kTile, stream));
  // Seeds from the k-NN lists (mutual reachability with alpha 1 only: there
  // a list edge's weight needs no distance).
  bool seeds = false;
  if constexpr (std::is_same<Weight, MutualReachWeight>::value)
    seeds = knn && knn->pos && weight.alpha == 1.0f && index.numInstances == 1;
  DeviceBuffer<unsigned long long> seed;
  if (seeds)
    CUHC_TRY(st, seed.allocate(n, stream));
  int numComponents = n, totalEdges = 0, rounds = 0;
  unsigned long long tilesSoFar = 0;
  int hostCounters[4];
  // Each instance of a batch ends as one component; padding slots stay
  // components of their own.
  const int finalComponents = index.numInstances + index.numPads;
  int maxJumps = 1;
  while ((1 << maxJumps) < n)
    ++maxJumps;
  // Radius proposal (single linkage, one instance, 16 features, a model
  // loaded) or training-row logging: per-round features of every position.
  const RadiusModel model = currentRadiusModel();
  const bool plainWeight = std::is_same<Weight, PlainWeight>::value;
  const bool useRadius = plainWeight && !radiusLog && model.params && index.d == kRadiusDims &&
                         index.numInstances == 1;
  const bool logRows = plainWeight && radiusLog && index.d == kRadiusDims &&
                       index.numInstances == 1;
  DeviceBuffer<float> features, prediction, radius, targets;
  DeviceBuffer<int> compSize;
  DeviceBuffer<unsigned long long> certified;
  if (useRadius || logRows) {
    CUHC_TRY(st, features.allocate((size_t)n * kRadiusFeatures, stream));
    CUHC_TRY(st, compSize.allocate(n, stream));
    CUHC_TRY(st, prediction.allocate(n, stream));
    CUHC_TRY(st, radius.allocate(n, stream));
    CUHC_TRY(st, targets.allocate(n, stream));
    CUHC_TRY(st, certified.allocate(4, stream)); // certified rows, then [mark, capped, fallback]
    CUHC_TRY(st, cudaMemsetAsync(certified.get(), 0, 4 * sizeof(unsigned long long), stream));
  }
  auto enqueueFeatures = [&](int round) {
    StatusChain fs;
    CUHC_TRY(fs, cudaMemsetAsync(compSize.get(), 0, n * sizeof(int), stream));
    radius_detail::componentSizes<<<blocks(n), 256, 0, stream>>>(comp.get(), index.order.get(), n,
                                                                 compSize.get());
    noteLaunch();
    radius_detail::radiusFeatures<<<blocks(n), 256, 0, stream>>>(
        index.tiled.get(), n, index.d, index.kc, index.tileFloats(), index.order.get(),
        index.nodeLow.get(), index.nodeHigh.get(), comp.get(), compSize.get(), nearest.get(),
        round, features.get());
    noteLaunch();
    CUHC_TRY(fs, cudaGetLastError());
    return fs.code;
  };
  std::mt19937_64 logRng(radiusLog ? radiusLog->seed : 0);
  unsigned long long proposedRows = 0;

  // One round, enqueued on the stream with no host work: counters[0] counts
  // every edge so far (edges are written at absolute slots), counters[1..2]
  // this round's roots and unjumped parents.
  auto enqueueRound = [&](bool first, int jumps, bool timed) {
    StatusChain rs;
    CUHC_TRY(rs, index.updatePurity(comp.get()));
    fillU32<<<blocks(n), 256, 0, stream>>>(compBest.get(), 0x7f800000u, n); noteLaunch();
    if (!first) {
      seedComponentBest<<<blocks(n), 256, 0, stream>>>(nearest.get(), index.rank.get(),
                                                       comp.get(), compBest.get(), n);
      noteLaunch();
    }
    if constexpr (std::is_same<Weight, MutualReachWeight>::value) {
      if (seeds) {
        seedFromKnn<<<blocks(n), 256, 0, stream>>>(knn->pos, knn->tie, knn->k, weight.value,
                                                   index.order.get(), comp.get(), seed.get(),
                                                   nearest.get(), compBest.get(), n);
        noteLaunch();
        p.seedKey = seed.get();
      }
    }
    if (screened) {
      packMeta<<<blocks(index.numTiles * kTile), 256, 0, stream>>>(
          index.order.get(), comp.get(), weight.value, n, index.numTiles, packed.get());
      noteLaunch();
      p.packedMeta = packed.get();
    }
    CUHC_TRY(rs, cudaGetLastError());
    p.singletons = first;
    p.radius = nullptr;
    // Heaviest row tiles first: by the last pass's work (boxes before any).
    CUHC_TRY(rs, index.orderTiles(!index.tileWorkValid, true));
    p.tileOrder = index.tileOrder.get();
    p.tileWork = index.tileWork.get();
    if (useRadius || logRows)
      CUHC_TRY(rs, enqueueFeatures(rounds));
    if (useRadius) {
      CUHC_TRY(rs, mlpForward(model.params, features.get(), n, prediction.get(), stream));
      radius_detail::radiusFromPrediction<<<blocks(n), 256, 0, stream>>>(
          prediction.get(), index.order.get(), n, model.offset, radius.get());
      noteLaunch();
      p.radius = radius.get();
      proposedRows += (unsigned long long)index.numPoints;
      radius_detail::radiusTileStep<<<1, 1, 0, stream>>>(tiles.get(), 0, certified.get() + 1);
      noteLaunch();
    }
    {
      PassTimer timer(timed ? (screened ? kTimerScreenPass : kTimerNearestPass) : -1, stream);
      if (screened)
        CUHC_TRY(rs, (launchScreen<Metric, Weight, false>(p, metric, weight, index.kc, stream)));
      else
        CUHC_TRY(rs, (launchPass<Metric, Weight, false>(p, metric, weight, index.kc, stream)));
      if (useRadius) {
        // Certify by component; the rest search again with no cap while
        // certified rows sit out. compBest already holds real edge weights
        // (seeds from the last round, and what rows published during the
        // pass); every row's final best goes in too, so it ends at most the
        // lightest edge found, which is what certification compares with.
        radius_detail::radiusTileStep<<<1, 1, 0, stream>>>(tiles.get(), 1, certified.get() + 1);
        noteLaunch();
        radius_detail::componentMinFound<<<blocks(n), 256, 0, stream>>>(
            nearest.get(), index.order.get(), comp.get(), n, compBest.get());
        noteLaunch();
        radius_detail::certifyRows<<<blocks(n), 256, 0, stream>>>(
            nearest.get(), index.order.get(), comp.get(), compBest.get(), n, radius.get(),
            certified.get());
        noteLaunch();
        if (screened)
          CUHC_TRY(rs, (launchScreen<Metric, Weight, false>(p, metric, weight, index.kc, stream)));
        else
          CUHC_TRY(rs, (launchPass<Metric, Weight, false>(p, metric, weight, index.kc, stream)));
        radius_detail::radiusTileStep<<<1, 1, 0, stream>>>(tiles.get(), 2, certified.get() + 1);
        noteLaunch();
        p.radius = nullptr;
      }
      if (timer.start) {
        unsigned long long tilesNow = 0;
        cudaMemcpyAsync(&tilesNow, tiles.get(), sizeof(tilesNow), cudaMemcpyDeviceToHost, stream);
        timer.finish(tilesNow - tilesSoFar);
        tilesSoFar = tilesNow;
      }
    }
    if (logRows) {
      radius_detail::radiusTargets<<<blocks(n), 256, 0, stream>>>(nearest.get(), index.order.get(),
                                                                  n, targets.get());
      noteLaunch();
      std::vector<float> hf((size_t)n * kRadiusFeatures), ht(n);
      CUHC_TRY(rs, cudaMemcpyAsync(hf.data(), features.get(), hf.size() * sizeof(float),
                                   cudaMemcpyDeviceToHost, stream));
      CUHC_TRY(rs, cudaMemcpyAsync(ht.data(), targets.get(), ht.size() * sizeof(float),
                                   cudaMemcpyDeviceToHost, stream));
      CUHC_TRY(rs, cudaStreamSynchronize(stream));
      std::vector<int> rows;
      for (int i = 0; i < n; ++i)
        if (std::isfinite(ht[i]))
          rows.push_back(i);
      std::shuffle(rows.begin(), rows.end(), logRng);
      rows.resize(std::min<size_t>(rows.size(), (size_t)radiusLog->maxRowsPerRound));
      for (const int i : rows) {
        radiusLog->features.insert(radiusLog->features.end(), hf.begin() + (size_t)i * kRadiusFeatures,
                                   hf.begin() + (size_t)(i + 1) * kRadiusFeatures);
        radiusLog->targets.push_back(ht[i]);
      }
    }
    index.tileWorkValid = true;
    CUHC_TRY(rs, cudaMemsetAsync(compKey.get(), 0xff, n * sizeof(unsigned long long), stream));
    CUHC_TRY(rs, cudaMemsetAsync(compV.get(), 0xff, n * sizeof(unsigned int), stream));
    CUHC_TRY(rs, cudaMemsetAsync(counters.get() + 1, 0, 2 * sizeof(int), stream));
    componentKeyPass1<<<blocks(n), 256, 0, stream>>>(nearest.get(), index.order.get(), comp.get(),
                                                     compKey.get(), n); noteLaunch();
    componentKeyPass2<<<blocks(n), 256, 0, stream>>>(nearest.get(), index.order.get(), comp.get(),
                                                     compKey.get(), compV.get(), n); noteLaunch();
    hookComponents<<<blocks(n), 256, 0, stream>>>(
        comp.get(), index.rank.get(), compKey.get(), compV.get(), parent.get(), edges.u.get(),
        edges.v.get(), edges.w.get(), counters.get(), n - 1, n); noteLaunch();
    for (int jmp = 0; jmp <= jumps; ++jmp) {
      jumpParents<<<blocks(n), 256, 0, stream>>>(comp.get(), parent.get(), n);
      noteLaunch();
    }
    countRoots<<<blocks(n), 256, 0, stream>>>(comp.get(), parent.get(), counters.get(), n); noteLaunch();
    relabel<<<blocks(n), 256, 0, stream>>>(comp.get(), parent.get(), n); noteLaunch();
    CUHC_TRY(rs, cudaGetLastError());
    return rs.code;
  };
  // Batches replay rounds after the first as one captured CUDA graph (the
  // round's launches and memsets with the largest jump count, extra jumps
  // being no-ops); timing needs events between launches and runs eagerly.
  const bool useGraph = index.numInstances > 1 && !timingEnabled();
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graphExec = nullptr;
  CUHC_TRY(st, cudaMemsetAsync(counters.get(), 0, 4 * sizeof(int), stream));
  while (st.ok() && numComponents > finalComponents) {
    if (useGraph && rounds > 0) {
      if (!graphExec) {
        CUHC_TRY(st, cudaStreamBeginCapture(stream, cudaStreamCaptureModeRelaxed));
        const int captured = enqueueRound(false, maxJumps, false);
        const cudaError_t ended = cudaStreamEndCapture(stream, &graph);
        CUHC_TRY(st, captured);
        CUHC_TRY(st, ended);
        CUHC_TRY(st, cudaGraphInstantiate(&graphExec, graph, 0));
        if (!st.ok())
          break;
      }
      CUHC_TRY(st, cudaGraphLaunch(graphExec, stream));
    } else {
      int jumps = 1;
      while ((1 << jumps) < numComponents)
        ++jumps;
      CUHC_TRY(st, enqueueRound(rounds == 0, jumps, true));
    }
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
    const int added = hostCounters[0] - totalEdges;
    if (hostCounters[2] != 0) {
      st(kErrorTimeout);
      break;
    }
    if (added == 0) {
      st(kErrorDisconnected);
      break;
    }
    totalEdges = hostCounters[0];
    numComponents = hostCounters[1];
    if (totalEdges > n - 1) {
      st(kErrorNonFinite);
      break;
    }
  }
  if (useRadius) {
    unsigned long long counts[4] = {};
    cudaMemcpyAsync(counts, certified.get(), sizeof(counts), cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    addRadiusStats(proposedRows, counts[0], counts[2], counts[3]);
  }
  if (graphExec)
    cudaGraphExecDestroy(graphExec);
  if (graph)
    cudaGraphDestroy(graph);
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
                  PassStats *stats, cudaStream_t stream, const int *coreRank, int *knnPos,
                  int *knnTie) {
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
  p.coreRank = coreRank;
  p.knnPos = knnPos;
  p.knnTie = knnTie;
  CUHC_TRY(st, index.orderTiles(!index.tileWorkValid));
  p.tileOrder = index.tileOrder.get();
  p.tileWork = index.tileWork.get();
  p.tilesComputed = tiles.get();
  p.error = error.get();
  p.screenStats = screenCounters();
  p.screenAudit = screenAuditWords();
  p.rootOfTile = index.numInstances > 1 ? index.rootOfTile.get() : nullptr;
  {
    const bool screened =
        useScreen<Metric>(index.d, k) && screenDataOk<Metric>(index);
    const ScreenShape shape =
        screened ? tunedScreenShape<Metric>(index, metric, k, core, stream) : ScreenShape{};
    ScreenShapeScope shapeScope(shape);
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
  index.tileWorkValid = true;
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

// Device milliseconds of the k-NN pass restricted to the first sampleTiles
// row tiles, screened or plain (the batched path's autotuner); writes the
// core distances of those rows only.
template <class Metric>
float timeKnnSample(SpatialIndex &index, const Metric &metric, int k, bool screened,
                    int sampleTiles, float *core, cudaStream_t stream) {
  PassParams p{};
  p.tiled = index.tiled.get();
  p.n = index.n;
  p.d = index.d;
  p.numChunks = index.numChunks;
  p.numTiles = std::min(sampleTiles, index.numTiles);
  p.order = index.order.get();
  p.nodeLeft = index.nodeLeft.get();
  p.nodeRight = index.nodeRight.get();
  p.nodeFirstTile = index.nodeFirstTile.get();
  p.leafOfTile = index.leafOfTile.get();
  p.nodeLow = index.nodeLow.get();
  p.nodeHigh = index.nodeHigh.get();
  p.prune = true;
  p.core = core;
  p.k = k;
  p.rootOfTile = index.numInstances > 1 ? index.rootOfTile.get() : nullptr;
  cudaEvent_t start, stop;
  cudaEventCreate(&start);
  cudaEventCreate(&stop);
  cudaEventRecord(start, stream);
  const int status =
      screened ? launchScreen<Metric, PlainWeight, true>(p, metric, PlainWeight{}, index.kc, stream)
               : launchPass<Metric, PlainWeight, true>(p, metric, PlainWeight{}, index.kc, stream);
  cudaEventRecord(stop, stream);
  cudaEventSynchronize(stop);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, start, stop);
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  return status == 0 ? ms : INFINITY;
}

// Whether this index's passes can run screened (metric, width, shared
// memory, data extent), ignoring the screen mode's "off".
template <class Metric> bool screenable(SpatialIndex &index, int k) {
  return useScreen<Metric>(index.d, k) && screenDataOk<Metric>(index);
}

// Pipeline-shape tuner of the screened k-NN pass: times candidate (ring
// slots, copy lead) pairs -- the most slots that fit with leads 2-6, and the
// fewest slots with lead 3 -- on the first 2 x SMs row tiles of the index
// (twice each, the faster kept) and returns the fastest, cached per process
// by (metric, d, k, batched or not). A shape changes time only, never a
// result. `scratch` receives throw-away core distances (n floats).
template <class Metric>
ScreenShape tunedScreenShape(SpatialIndex &index, const Metric &m, int k, float *scratch,
                             cudaStream_t s) {
  static std::mutex mutex;
  static std::map<std::tuple<size_t, int, int, bool>, ScreenShape> tuned;
  const auto key = std::make_tuple(typeid(Metric).hash_code(), index.d, k, index.numInstances > 1);
  {
    std::lock_guard<std::mutex> lock(mutex);
    const auto it = tuned.find(key);
    if (it != tuned.end())
      return it->second;
  }
  const int maxStages = screenStagesFor(index.d, k);
  std::vector<ScreenShape> candidates;
  for (int lead = 2; lead <= 6; ++lead)
    if (lead <= maxStages - 1)
      candidates.push_back(ScreenShape{maxStages, lead});
  if (maxStages > kScreenMinStages)
    candidates.push_back(ScreenShape{kScreenMinStages, 3});
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  ScreenShape best{};
  float bestMs = INFINITY;
  for (const ScreenShape shape : candidates) {
    ScreenShapeScope scope(shape);
    float ms = INFINITY;
    for (int rep = 0; rep < 2; ++rep)
      ms = std::min(ms, timeKnnSample(index, m, k, true, 2 * sms, scratch, s));
    if (ms < bestMs) {
      bestMs = ms;
      best = shape;
    }
  }
  std::lock_guard<std::mutex> lock(mutex);
  tuned[key] = best;
  return best;
}

} // namespace cuhc
