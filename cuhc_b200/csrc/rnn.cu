// Ward linkage by rounds of reciprocal nearest neighbours (RNN), on the
// shared pass engine.
//
// Each round: one all-pairs nearest pass over the active clusters' centroids
// with the Ward selection weight (every cluster its own component); every
// pair of clusters that are each other's nearest merges, all at once; the
// survivors are compacted for the next round. Same algorithm and formulas as
// the reference (rnn_ward.cuh:248-368), with its hand-over rule to a dense or
// chain tail when a round merges less than minProgress of the clusters.
//
// Clusters are stored in k-d order (for pruning) but every decision uses the
// cluster's representative, its smallest original point index: the packed
// keys carry it, ties go to the lower one, and the merged centroid is formed
// from the lower-representative cluster. Without pruning the reference keeps
// its slots in representative order (compaction preserves it), so this is
// the reference's arithmetic bit for bit, whatever the physical order.
#include "profiling.cuh"
#include "rnn.cuh"

#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <vector>

#include "metrics.cuh"
#include "passes.cuh"
#include "screen.cuh"

namespace cuhc {

int chainOnClusters(const float *centroids, const int *sizes, int m, int d, cudaStream_t s,
                    std::vector<int> &a, std::vector<int> &b, std::vector<float> &h);
int denseOnWardMatrix(const float *centroids, const int *sizes, const int *reps, int m, int d,
                      int numPoints, cudaStream_t s, std::vector<int> &u, std::vector<int> &v,
                      std::vector<float> &h);
int denseLinkageFromMatrix(float *distances, const int *initialSize, const int *initialId,
                           int firstNewId, int m, int linkageId, double *deviceTree,
                           cudaStream_t s);

namespace {

inline int blocks(long long work, int threads = 256) { return (int)((work + threads - 1) / threads); }

// Ward distance squared from the squared distance of two centroids, in the
// reference's operation order (rnn_ward.cuh:45-48).
__device__ __forceinline__ float wardFromSquared(float squared, float si, float sj) {
  return 2.0f * (si * sj) / (si + sj) * squared;
}

__global__ void initClusters(const int *__restrict__ order, int n, int *__restrict__ size,
                             float *__restrict__ sizeF, int *__restrict__ rep,
                             int *__restrict__ slotOfRep) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  size[i] = 1;
  sizeF[i] = 1.0f;
  rep[i] = order[i];
  slotOfRep[order[i]] = i;
}

// Positions -> row-major centroids in position order.
__global__ void gatherRows(const float *__restrict__ points, const int *__restrict__ order, int n,
                           int d, float *__restrict__ out) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)n * d)
    return;
  const int i = (int)(e / d), f = (int)(e % d);
  out[e] = points[(size_t)order[i] * d + f];
}

// partner[i]: the slot that i pairs with this round, or -1; survive[i] = 0
// if i is absorbed into a partner with a lower representative.
__global__ void rnnPartners(const unsigned long long *__restrict__ nearest,
                            const int *__restrict__ slotOfRep, const int *__restrict__ rep, int m,
                            int *__restrict__ partner, int *__restrict__ survive) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m)
    return;
  const unsigned long long key = nearest[i];
  int j = -1;
  if (key != kEmptyKey) {
    const int cand = slotOfRep[keyIndex(key)];
    const unsigned long long back = nearest[cand];
    if (back != kEmptyKey && (int)keyIndex(back) == rep[i])
      j = cand;
  }
  partner[i] = j;
  survive[i] = !(j >= 0 && rep[j] < rep[i]);
}

// Next round's clusters: slot i (not absorbed) goes to newIndex[i]; with a
// partner j its centroid is c_i + (c_j - c_i) * n_j / (n_i + n_j), the
// reference's incremental form (exact for equal centroids), and the merge is
// recorded with the exact height sqrt(ward(|c_i - c_j|^2)).
__global__ void rnnMerge(const float *__restrict__ cent, const int *__restrict__ size,
                         const int *__restrict__ rep, const int *__restrict__ partner,
                         const int *__restrict__ newIndex, int m, int d, float *__restrict__ nextCent,
                         int *__restrict__ nextSize, float *__restrict__ nextSizeF,
                         int *__restrict__ nextRep, int *__restrict__ slotOfRep,
                         int *__restrict__ mergeU, int *__restrict__ mergeV,
                         float *__restrict__ mergeH, int *__restrict__ mergeCount, int capacity) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)m * d)
    return;
  const int i = (int)(e / d), f = (int)(e % d);
  const int j = partner[i];
  if (j >= 0 && rep[j] < rep[i])
    return;
  const int to = newIndex[i];
  const float ci = cent[e];
  float c = ci;
  const float si = (float)size[i];
  if (j >= 0) {
    const float sj = (float)size[j];
    c = fmaf(cent[(size_t)j * d + f] - ci, sj / (si + sj), ci);
  }
  nextCent[(size_t)to * d + f] = c;
  if (f == 0) {
    const int merged = size[i] + (j >= 0 ? size[j] : 0);
    nextSize[to] = merged;
    nextSizeF[to] = (float)merged;
    nextRep[to] = rep[i];
    slotOfRep[rep[i]] = to;
    if (j >= 0) {
      const float *a = cent + (size_t)i * d, *b = cent + (size_t)j * d;
      float squared = 0.0f;
      for (int k = 0; k < d; ++k) {
        const float diff = a[k] - b[k];
        squared = fmaf(diff, diff, squared);
      }
      const int slot = atomicAdd(mergeCount, 1);
      if (slot < capacity) {
        mergeU[slot] = min(rep[i], rep[j]);
        mergeV[slot] = max(rep[i], rep[j]);
        mergeH[slot] = sqrtf(wardFromSquared(squared, si, (float)size[j]));
      }
    }
  }
}

__global__ void gatherClusters(const int *__restrict__ perm, const float *__restrict__ cent,
                               const int *__restrict__ size, int m, int d,
                               float *__restrict__ outCent, int *__restrict__ outSize) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)m * d)
    return;
  const int i = (int)(e / d), f = (int)(e % d);
  outCent[e] = cent[(size_t)perm[i] * d + f];
  if (f == 0)
    outSize[i] = size[perm[i]];
}

bool lessEdge(float wa, int ua, int va, float wb, int ub, int vb) {
  if (wa != wb)
    return wa < wb;
  if (ua != ub)
    return ua < ub;
  return va < vb;
}

struct Merge {
  int u, v;
  float w;
};

// Chain-order merges -> tree order: heights made non-decreasing up the tree
// (a merge at least as high as the merges below it), then a stable sort by
// height, as the reference's orderChainMerges (nn_chain.cuh:178-188).
void orderChainMerges(std::vector<Merge> &merges, int n) {
  std::vector<int> parent(n);
  std::vector<float> height(n, 0.0f);
  for (int i = 0; i < n; ++i)
    parent[i] = i;
  auto find = [&](int x) {
    while (parent[x] != x) {
      parent[x] = parent[parent[x]];
      x = parent[x];
    }
    return x;
  };
  for (Merge &mg : merges) {
    const int ru = find(mg.u), rv = find(mg.v);
    mg.w = std::max({mg.w, height[ru], height[rv]});
    parent[rv] = ru;
    height[ru] = mg.w;
  }
  std::stable_sort(merges.begin(), merges.end(),
                   [](const Merge &x, const Merge &y) { return x.w < y.w; });
}

bool wardMatrixFits(int m) {
  size_t freeBytes = 0, total = 0;
  if (cudaMemGetInfo(&freeBytes, &total) != cudaSuccess)
    return false;
  return 4.0 * m * m <= 0.9 * (double)freeBytes;
}

} // namespace

int rnnWard(const float *devPoints, int n, int d, const RnnOptions &options, double *hostTree,
            PassStats *stats, cudaStream_t s) {
  if (n < 2)
    return 0;
  StatusChain st;
  const int mode = currentPruneMode();
  const bool prune = mode != 2 && d <= 256 && numTilesFor(n) >= 2;
  SpatialIndex index;
  CUHC_TRY(st, index.build(devPoints, n, d, prune, s));
  DeviceBuffer<float> cent[2], sizeF[2];
  DeviceBuffer<int> size[2], rep[2];
  DeviceBuffer<int> slotOfRep, partner, survive, newIndex, counter, error;
  DeviceBuffer<int> mergeU, mergeV;
  DeviceBuffer<float> mergeH;
  DeviceBuffer<unsigned long long> nearest, tiles;
  for (int b = 0; b < 2; ++b) {
    CUHC_TRY(st, cent[b].allocate((size_t)n * d, s));
    CUHC_TRY(st, sizeF[b].allocate(paddedToTiles(n), s));
    CUHC_TRY(st, size[b].allocate(n, s));
    CUHC_TRY(st, rep[b].allocate(paddedToTiles(n), s));
  }
  CUHC_TRY(st, slotOfRep.allocate(n, s));
  CUHC_TRY(st, partner.allocate(n, s));
  CUHC_TRY(st, survive.allocate(n, s));
  CUHC_TRY(st, newIndex.allocate(n, s));
  CUHC_TRY(st, counter.allocate(1, s));
  CUHC_TRY(st, error.allocate(1, s));
  CUHC_TRY(st, mergeU.allocate(n - 1, s));
  CUHC_TRY(st, mergeV.allocate(n - 1, s));
  CUHC_TRY(st, mergeH.allocate(n - 1, s));
  CUHC_TRY(st, nearest.allocate(n, s));
  CUHC_TRY(st, tiles.allocate(1, s));
  size_t scanBytes = 0;
  CUHC_TRY(st, cub::DeviceScan::ExclusiveSum(nullptr, scanBytes, survive.get(), newIndex.get(),
                                             n, s));
  DeviceBuffer<unsigned char> scanTemp;
  CUHC_TRY(st, scanTemp.allocate(scanBytes, s));
  if (!st.ok())
    return st.code;
  CUHC_TRY(st, cudaMemsetAsync(counter.get(), 0, sizeof(int), s));
  CUHC_TRY(st, cudaMemsetAsync(error.get(), 0, sizeof(int), s));
  CUHC_TRY(st, cudaMemsetAsync(tiles.get(), 0, sizeof(unsigned long long), s));
  initClusters<<<blocks(n), 256, 0, s>>>(index.order.get(), n, size[0].get(), sizeF[0].get(),
                                         rep[0].get(), slotOfRep.get());
  noteLaunch();
  gatherRows<<<blocks((long long)n * d), 256, 0, s>>>(devPoints, index.order.get(), n, d,
                                                      cent[0].get());
  noteLaunch();
  CUHC_TRY(st, cudaGetLastError());

  std::vector<int> roundEnd;
  int m = n, merged = 0, cur = 0, rounds = 0;
  enum { kNone, kDense, kChain } tail = kNone;
  unsigned long long tilesSoFar = 0;
  while (st.ok() && m > 1) {
    if (options.allowDense && m <= options.denseBelow && wardMatrixFits(m)) {
      tail = kDense;
      break;
    }
    if (rounds > 0)
      CUHC_TRY(st, index.retile(cent[cur].get(), m));
    CUHC_TRY(st, index.updateMinValues(sizeF[cur].get()));
    PassParams p{};
    p.tiled = index.tiled.get();
    p.n = m;
    p.d = d;
    p.numChunks = index.numChunks;
    p.numTiles = index.numTiles;
    p.order = rep[cur].get();
    p.component = nullptr;
    p.nodeLeft = index.nodeLeft.get();
    p.nodeRight = index.nodeRight.get();
    p.nodeFirstTile = index.nodeFirstTile.get();
    p.leafOfTile = index.leafOfTile.get();
    p.nodePure = nullptr;
    p.nodeLow = index.nodeLow.get();
    p.nodeHigh = index.nodeHigh.get();
    p.nodeMinValue = index.nodeMinValue.get();
    p.prune = prune;
    p.nearest = nearest.get();
    p.compBest = nullptr;
    p.tilesComputed = tiles.get();
    p.error = error.get();
  p.screenStats = screenCounters();
  p.screenAudit = screenAuditWords();
    WardWeight w;
    w.value = sizeF[cur].get();
    {
      const bool screened =
          useScreen<SqEuclideanMetric>(d, 0) && index.extentsWithin(kScreenMaxExtent);
      PassTimer timer(screened ? kTimerScreenPass : kTimerNearestPass, s);
      if (screened)
        CUHC_TRY(st, (launchScreen<SqEuclideanMetric, WardWeight, false>(
                         p, SqEuclideanMetric{}, w, index.kc, s)));
      else
        CUHC_TRY(st, (launchPass<SqEuclideanMetric, WardWeight, false>(p, SqEuclideanMetric{}, w,
                                                                       index.kc, s)));
      if (timer.start) {
        unsigned long long now = 0;
        cudaMemcpyAsync(&now, tiles.get(), sizeof(now), cudaMemcpyDeviceToHost, s);
        timer.finish(now - tilesSoFar);
        tilesSoFar = now;
      }
    }
    rnnPartners<<<blocks(m), 256, 0, s>>>(nearest.get(), slotOfRep.get(), rep[cur].get(), m,
                                          partner.get(), survive.get());
    noteLaunch();
    CUHC_TRY(st, cub::DeviceScan::ExclusiveSum(scanTemp.get(), scanBytes, survive.get(),
                                               newIndex.get(), m, s));
    const int nxt = 1 - cur;
    rnnMerge<<<blocks((long long)m * d), 256, 0, s>>>(
        cent[cur].get(), size[cur].get(), rep[cur].get(), partner.get(), newIndex.get(), m, d,
        cent[nxt].get(), size[nxt].get(), sizeF[nxt].get(), rep[nxt].get(), slotOfRep.get(),
        mergeU.get(), mergeV.get(), mergeH.get(), counter.get(), n - 1);
    noteLaunch();
    CUHC_TRY(st, cudaGetLastError());
    int total = 0, passError = 0;
    CUHC_TRY(st, cudaMemcpyAsync(&total, counter.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CUHC_TRY(st, cudaMemcpyAsync(&passError, error.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    CUHC_TRY(st, cudaStreamSynchronize(s));
    if (!st.ok())
      break;
    if (passError != 0) {
      st(passError);
      break;
    }
    ++rounds;
    const int roundMerges = total - merged;
    merged = total;
    roundEnd.push_back(total);
    cur = nxt;
    const int before = m;
    m -= roundMerges;
    if (merged > n - 1) {
      st(kErrorNonFinite);
      break;
    }
    if (m > 1 && (roundMerges == 0 || roundMerges < options.minProgress * before)) {
      tail = options.allowDense && wardMatrixFits(m) ? kDense : kChain;
      break;
    }
  }
  int err = 0;
  CUHC_TRY(st, cudaMemcpyAsync(&err, error.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
  unsigned long long tileCount = 0;
  CUHC_TRY(st, cudaMemcpyAsync(&tileCount, tiles.get(), sizeof(tileCount),
                               cudaMemcpyDeviceToHost, s));
  std::vector<int> hu(merged), hv(merged);
  std::vector<float> hh(merged);
  if (merged > 0) {
    CUHC_TRY(st, cudaMemcpyAsync(hu.data(), mergeU.get(), merged * sizeof(int),
                                 cudaMemcpyDeviceToHost, s));
    CUHC_TRY(st, cudaMemcpyAsync(hv.data(), mergeV.get(), merged * sizeof(int),
                                 cudaMemcpyDeviceToHost, s));
    CUHC_TRY(st, cudaMemcpyAsync(hh.data(), mergeH.get(), merged * sizeof(float),
                                 cudaMemcpyDeviceToHost, s));
  }
  CUHC_TRY(st, cudaStreamSynchronize(s));
  if (err)
    st(err);
  if (stats) {
    stats->tilesComputed += tileCount;
    stats->passes += rounds;
    for (int r = 0, mm = n; r < rounds; ++r) {
      const int t = numTilesFor(mm);
      stats->tilesTotal += (unsigned long long)t * t;
      mm -= roundEnd[r] - (r ? roundEnd[r - 1] : 0);
    }
  }
  if (!st.ok())
    return st.code;

  std::vector<Merge> merges(merged);
  for (int i = 0; i < merged; ++i)
    merges[i] = Merge{hu[i], hv[i], hh[i]};
  // Within a round merges arrive in atomic order; sorting each round by the
  // edge order makes the result independent of scheduling.
  for (size_t r = 0; r < roundEnd.size(); ++r)
    std::sort(merges.begin() + (r == 0 ? 0 : roundEnd[r - 1]), merges.begin() + roundEnd[r],
              [](const Merge &x, const Merge &y) { return lessEdge(x.w, x.u, x.v, y.w, y.u, y.v); });

  if (tail != kNone && m > 1) {
    // The remaining clusters in representative order (the reference's slot
    // order), so the tails see the same slots.
    DeviceBuffer<int> keysOut, perm, permOut, tSize, repSorted;
    DeviceBuffer<float> tCent;
    CUHC_TRY(st, keysOut.allocate(m, s));
    CUHC_TRY(st, perm.allocate(m, s));
    CUHC_TRY(st, permOut.allocate(m, s));
    CUHC_TRY(st, tSize.allocate(m, s));
    CUHC_TRY(st, tCent.allocate((size_t)m * d, s));
    std::vector<int> iota(m);
    for (int i = 0; i < m; ++i)
      iota[i] = i;
    CUHC_TRY(st, cudaMemcpyAsync(perm.get(), iota.data(), m * sizeof(int),
                                 cudaMemcpyHostToDevice, s));
    size_t sortBytes = 0;
    CUHC_TRY(st, cub::DeviceRadixSort::SortPairs(nullptr, sortBytes, rep[cur].get(),
                                                 keysOut.get(), perm.get(), permOut.get(), m, 0,
                                                 32, s));
    DeviceBuffer<unsigned char> sortTemp;
    CUHC_TRY(st, sortTemp.allocate(sortBytes, s));
    CUHC_TRY(st, cub::DeviceRadixSort::SortPairs(sortTemp.get(), sortBytes, rep[cur].get(),
                                                 keysOut.get(), perm.get(), permOut.get(), m, 0,
                                                 32, s));
    gatherClusters<<<blocks((long long)m * d), 256, 0, s>>>(permOut.get(), cent[cur].get(),
                                                            size[cur].get(), m, d, tCent.get(),
                                                            tSize.get());
    noteLaunch();
    CUHC_TRY(st, cudaGetLastError());
    std::vector<int> reps(m);
    CUHC_TRY(st, cudaMemcpyAsync(reps.data(), keysOut.get(), m * sizeof(int),
                                 cudaMemcpyDeviceToHost, s));
    CUHC_TRY(st, cudaStreamSynchronize(s));
    std::vector<int> tu, tv;
    std::vector<float> th;
    if (tail == kDense) {
      CUHC_TRY(st, denseOnWardMatrix(tCent.get(), tSize.get(), keysOut.get(), m, d, n, s, tu, tv,
                                     th));
      for (size_t i = 0; i < tu.size(); ++i)
        merges.push_back(Merge{std::min(tu[i], tv[i]), std::max(tu[i], tv[i]), th[i]});
    } else {
      CUHC_TRY(st, chainOnClusters(tCent.get(), tSize.get(), m, d, s, tu, tv, th));
      for (size_t i = 0; i < tu.size(); ++i) {
        const int a = reps[tu[i]], b = reps[tv[i]];
        merges.push_back(Merge{std::min(a, b), std::max(a, b), th[i]});
      }
    }
    if (!st.ok())
      return st.code;
  }
  std::vector<int> u(merges.size()), v(merges.size());
  std::vector<float> h(merges.size());
  for (size_t i = 0; i < merges.size(); ++i) {
    u[i] = merges[i].u;
    v[i] = merges[i].v;
    h[i] = merges[i].w;
  }
  if (!mergesFormTree(u, v, h, n))
    return kErrorNonFinite;
  orderChainMerges(merges, n);
  for (size_t i = 0; i < merges.size(); ++i) {
    u[i] = merges[i].u;
    v[i] = merges[i].v;
    h[i] = merges[i].w;
  }
  treeFromOrderedMerges(u, v, h, n, hostTree);
  return 0;
}

int nnChainWard(const float *devPoints, int n, int d, double *hostTree, cudaStream_t s) {
  if (n < 2)
    return 0;
  StatusChain st;
  DeviceBuffer<int> ones;
  CUHC_TRY(st, ones.allocate(n, s));
  std::vector<int> hostOnes(n, 1);
  CUHC_TRY(st, cudaMemcpyAsync(ones.get(), hostOnes.data(), n * sizeof(int),
                               cudaMemcpyHostToDevice, s));
  std::vector<int> a, b;
  std::vector<float> h;
  CUHC_TRY(st, chainOnClusters(devPoints, ones.get(), n, d, s, a, b, h));
  if (!st.ok())
    return st.code;
  std::vector<Merge> merges(a.size());
  std::vector<int> u(a.size()), v(a.size());
  for (size_t i = 0; i < a.size(); ++i) {
    merges[i] = Merge{std::min(a[i], b[i]), std::max(a[i], b[i]), h[i]};
    u[i] = merges[i].u;
    v[i] = merges[i].v;
  }
  if (!mergesFormTree(u, v, h, n))
    return kErrorNonFinite;
  orderChainMerges(merges, n);
  for (size_t i = 0; i < merges.size(); ++i) {
    u[i] = merges[i].u;
    v[i] = merges[i].v;
    h[i] = merges[i].w;
  }
  treeFromOrderedMerges(u, v, h, n, hostTree);
  return 0;
}

} // namespace cuhc
