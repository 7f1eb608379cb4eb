// Agglomerative clustering on the dense n x n float32 distance matrix
// (algorithm "dense": complete / average linkage, any linkage on request,
// and the dense tail of the RNN rounds).
//
// Clusters live in matrix slots; merging slots a < b keeps the cluster in a.
// Every active slot caches its nearest active slot, so one merge is: the
// argmin of the cache (ties to the lower slot), a Lance-Williams update of
// row / column a in double, and a rescan of the rows whose cached nearest
// was a or b and got farther. The reference does the same three steps per
// merge (linkage.cuh:86-268) with the same tie rules and formulas.
//
// B200 shape: the three kernels of a step are captured once into a CUDA
// graph of kStepsPerGraph steps; the step counter lives on the device, so the
// graph is replayed ceil((n-1) / kStepsPerGraph) times with no host work in
// between and surplus steps exit at once.
#include "profiling.cuh"
#include "rnn.cuh"

#include <vector>

#include "metrics.cuh"
#include "pairwise.cuh"

namespace cuhc {

int pairwiseIntoMatrix(const float *points, int n, int d, int metricId, float p, float *out,
                       cudaStream_t s);

namespace {

constexpr int kReduceThreads = 1024, kRescanThreads = 256, kStepsPerGraph = 64;
enum LinkageKind : int { kSingleL = 0, kCompleteL = 1, kAverageL = 2, kWardL = 3 };

struct MergeRecord {
  int a, b;
  float distance;
  int sizeA, sizeB;
};

struct DenseState {
  float *dist;
  float *nearDist;
  int *nearSlot, *size, *id, *rescan, *rescanCount, *step;
  unsigned char *active;
  MergeRecord *merge;
  double *tree;
  int n, firstNewId, linkage;
};

// Distance from the merged cluster (a u b) to k from the old distances, in
// double (O(n) per merge; rounding would compound over thousands of merges).
__device__ double lanceWilliams(int linkage, double dak, double dbk, double dab, double na,
                                double nb, double nk) {
  switch (linkage) {
  case kSingleL:
    return fmin(dak, dbk);
  case kCompleteL:
    return fmax(dak, dbk);
  case kAverageL:
    return (na * dak + nb * dbk) / (na + nb);
  default: {
    // Ward on Euclidean (not squared) distances, as scipy and sklearn.
    const double t = na + nb + nk;
    const double sq = ((na + nk) * dak * dak + (nb + nk) * dbk * dbk - nk * dab * dab) / t;
    return sqrt(fmax(sq, 0.0));
  }
  }
}

__device__ __forceinline__ bool lessLoc(float da, int ia, float db, int ib) {
  return da < db || (da == db && ia < ib);
}

__global__ void denseInit(DenseState s, const int *initialSize, const int *initialId) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n)
    return;
  s.dist[(size_t)i * s.n + i] = INFINITY;
  s.size[i] = initialSize ? initialSize[i] : 1;
  s.id[i] = initialId ? initialId[i] : i;
  s.active[i] = 1;
  s.rescan[i] = i;
  if (i == 0) {
    *s.rescanCount = s.n;
    *s.step = 0;
  }
}

// Nearest active slot of every listed row (retired columns hold +inf).
__global__ void __launch_bounds__(kRescanThreads) denseRescan(DenseState s) {
  if (*s.step >= s.n - 1 && s.n > 1 && *s.step > 0) // past the last merge
    return;
  __shared__ float wd[kRescanThreads / 32];
  __shared__ int ws[kRescanThreads / 32];
  const int count = *s.rescanCount;
  for (int item = blockIdx.x; item < count; item += gridDim.x) {
    const int row = s.rescan[item];
    const float *r = s.dist + (size_t)row * s.n;
    float best = INFINITY;
    int slot = 0x7fffffff;
    for (int c = threadIdx.x; c < s.n; c += kRescanThreads)
      if (lessLoc(r[c], c, best, slot)) {
        best = r[c];
        slot = c;
      }
    for (int off = 16; off > 0; off /= 2) {
      const float od = __shfl_xor_sync(0xffffffffu, best, off);
      const int os = __shfl_xor_sync(0xffffffffu, slot, off);
      if (lessLoc(od, os, best, slot)) {
        best = od;
        slot = os;
      }
    }
    if ((threadIdx.x & 31) == 0) {
      wd[threadIdx.x >> 5] = best;
      ws[threadIdx.x >> 5] = slot;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < kRescanThreads / 32; ++w)
        if (lessLoc(wd[w], ws[w], best, slot)) {
          best = wd[w];
          slot = ws[w];
        }
      s.nearDist[row] = best;
      s.nearSlot[row] = slot;
    }
    __syncthreads();
  }
}

// One block: the closest pair, the tree row, the bookkeeping of slot a.
__global__ void __launch_bounds__(kReduceThreads) denseClosestPair(DenseState s) {
  const int step = *s.step;
  if (step >= s.n - 1)
    return;
  __shared__ float wd[kReduceThreads / 32];
  __shared__ int ws[kReduceThreads / 32];
  float best = INFINITY;
  int slot = 0x7fffffff;
  for (int i = threadIdx.x; i < s.n; i += kReduceThreads)
    if (lessLoc(s.nearDist[i], i, best, slot)) {
      best = s.nearDist[i];
      slot = i;
    }
  for (int off = 16; off > 0; off /= 2) {
    const float od = __shfl_xor_sync(0xffffffffu, best, off);
    const int os = __shfl_xor_sync(0xffffffffu, slot, off);
    if (lessLoc(od, os, best, slot)) {
      best = od;
      slot = os;
    }
  }
  if ((threadIdx.x & 31) == 0) {
    wd[threadIdx.x >> 5] = best;
    ws[threadIdx.x >> 5] = slot;
  }
  __syncthreads();
  if (threadIdx.x != 0)
    return;
  for (int w = 1; w < kReduceThreads / 32; ++w)
    if (lessLoc(wd[w], ws[w], best, slot)) {
      best = wd[w];
      slot = ws[w];
    }
  if (!(best < INFINITY) || slot < 0 || slot >= s.n) { // no finite pair left: stop
    *s.step = s.n;
    return;
  }
  const int other = s.nearSlot[slot];
  const int a = min(slot, other), b = max(slot, other);
  const int na = s.size[a], nb = s.size[b];
  const int ia = s.id[a], ib = s.id[b];
  *s.merge = MergeRecord{a, b, best, na, nb};
  double *row = s.tree + (size_t)step * 4;
  row[0] = min(ia, ib);
  row[1] = max(ia, ib);
  row[2] = best;
  row[3] = na + nb;
  s.size[a] = na + nb;
  s.id[a] = s.firstNewId + step;
  s.active[b] = 0;
  s.nearDist[b] = INFINITY;
  *s.rescanCount = 0;
}

// One thread per slot k: the Lance-Williams distance of the merged cluster,
// and whether k's cached nearest is still valid.
__global__ void denseMerge(DenseState s) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int step = *s.step;
  if (k >= s.n || step >= s.n - 1 || !s.active[k])
    return;
  const MergeRecord mg = *s.merge;
  const int a = mg.a, b = mg.b;
  const size_t n = s.n;
  if (k == a) {
    s.dist[(size_t)a * n + b] = INFINITY;
    s.rescan[atomicAdd(s.rescanCount, 1)] = a;
    return;
  }
  const float nd = (float)lanceWilliams(s.linkage, s.dist[(size_t)a * n + k],
                                        s.dist[(size_t)b * n + k], mg.distance, mg.sizeA,
                                        mg.sizeB, s.size[k]);
  s.dist[(size_t)a * n + k] = nd;
  s.dist[(size_t)k * n + a] = nd;
  s.dist[(size_t)k * n + b] = INFINITY;
  const int near = s.nearSlot[k];
  if (near == a || near == b) {
    if (nd <= s.nearDist[k]) {
      s.nearDist[k] = nd;
      s.nearSlot[k] = a;
    } else {
      s.rescan[atomicAdd(s.rescanCount, 1)] = k;
    }
  } else if (nd < s.nearDist[k]) {
    s.nearDist[k] = nd;
    s.nearSlot[k] = a;
  }
}

// Next step; stays at n - 1 after the last merge, and at n after an early
// stop (no finite pair left), which the host reports as an error.
__global__ void denseAdvance(DenseState s) {
  if (*s.step < s.n - 1)
    ++*s.step;
}

__global__ void wardTransform(float *dist, const int *size, int m) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)m * m)
    return;
  const int i = (int)(e / m), j = (int)(e % m);
  const float si = (float)size[i], sj = (float)size[j];
  dist[e] = sqrtf(2.0f * (si * sj) / (si + sj) * dist[e]);
}

} // namespace

int denseLinkageFromMatrix(float *distances, const int *initialSize, const int *initialId,
                           int firstNewId, int m, int linkageId, double *deviceTree,
                           cudaStream_t s) {
  if (m < 2)
    return 0;
  StatusChain st;
  DeviceBuffer<float> nearDist;
  DeviceBuffer<int> ints;
  DeviceBuffer<unsigned char> active;
  DeviceBuffer<MergeRecord> merge;
  CUHC_TRY(st, nearDist.allocate(m, s));
  CUHC_TRY(st, ints.allocate((size_t)4 * m + 2, s));
  CUHC_TRY(st, active.allocate(m, s));
  CUHC_TRY(st, merge.allocate(1, s));
  if (!st.ok())
    return st.code;
  DenseState ds{};
  ds.dist = distances;
  ds.nearDist = nearDist.get();
  ds.nearSlot = ints.get();
  ds.size = ints.get() + m;
  ds.id = ints.get() + 2 * m;
  ds.rescan = ints.get() + 3 * m;
  ds.rescanCount = ints.get() + 4 * m;
  ds.step = ints.get() + 4 * m + 1;
  ds.active = active.get();
  ds.merge = merge.get();
  ds.tree = deviceTree;
  ds.n = m;
  ds.firstNewId = firstNewId;
  ds.linkage = linkageId;
  const int perSlot = (m + 255) / 256;
  int device = 0, sms = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  denseInit<<<perSlot, 256, 0, s>>>(ds, initialSize, initialId);
  noteLaunch();
  denseRescan<<<4 * sms, kRescanThreads, 0, s>>>(ds);
  noteLaunch();
  CUHC_TRY(st, cudaGetLastError());
  // One graph of kStepsPerGraph merges, replayed.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  CUHC_TRY(st, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  if (st.ok()) {
    for (int i = 0; i < kStepsPerGraph; ++i) {
      denseClosestPair<<<1, kReduceThreads, 0, s>>>(ds);
      denseMerge<<<perSlot, 256, 0, s>>>(ds);
      denseRescan<<<4 * sms, kRescanThreads, 0, s>>>(ds);
      denseAdvance<<<1, 1, 0, s>>>(ds);
    }
    CUHC_TRY(st, cudaStreamEndCapture(s, &graph));
  }
  CUHC_TRY(st, cudaGraphInstantiate(&exec, graph, 0));
  const int replays = (m - 1 + kStepsPerGraph - 1) / kStepsPerGraph;
  for (int r = 0; r < replays && st.ok(); ++r) {
    CUHC_TRY(st, cudaGraphLaunch(exec, s));
    noteLaunch(4 * kStepsPerGraph);
  }
  CUHC_TRY(st, cudaStreamSynchronize(s));
  if (exec)
    cudaGraphExecDestroy(exec);
  if (graph)
    cudaGraphDestroy(graph);
  int step = 0;
  CUHC_TRY(st, cudaMemcpy(&step, ds.step, sizeof(int), cudaMemcpyDeviceToHost));
  if (st.ok() && step != m - 1)
    st(kErrorNonFinite);
  return st.code;
}

int denseLinkage(const float *devPoints, int n, int d, int metricId, float p, int linkageId,
                 double *hostTree, cudaStream_t s) {
  if (n < 2)
    return 0;
  StatusChain st;
  DeviceBuffer<float> dist;
  DeviceBuffer<double> tree;
  CUHC_TRY(st, dist.allocate((size_t)n * n, s));
  CUHC_TRY(st, tree.allocate((size_t)(n - 1) * 4, s));
  CUHC_TRY(st, pairwiseIntoMatrix(devPoints, n, d, metricId, p, dist.get(), s));
  CUHC_TRY(st, denseLinkageFromMatrix(dist.get(), nullptr, nullptr, n, n, linkageId, tree.get(), s));
  CUHC_TRY(st, cudaMemcpyAsync(hostTree, tree.get(), tree.bytes(), cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaStreamSynchronize(s));
  return st.code;
}

int denseOnWardMatrix(const float *centroids, const int *sizes, const int *reps, int m, int d,
                      int numPoints, cudaStream_t s, std::vector<int> &u, std::vector<int> &v,
                      std::vector<float> &h) {
  StatusChain st;
  DeviceBuffer<float> dist;
  DeviceBuffer<double> tree;
  CUHC_TRY(st, dist.allocate((size_t)m * m, s));
  CUHC_TRY(st, tree.allocate((size_t)(m - 1) * 4, s));
  CUHC_TRY(st, pairwiseIntoMatrix(centroids, m, d, kSqEuclidean, 2.0f, dist.get(), s));
  wardTransform<<<(int)(((long long)m * m + 255) / 256), 256, 0, s>>>(dist.get(), sizes, m);
  noteLaunch();
  CUHC_TRY(st, cudaGetLastError());
  CUHC_TRY(st, denseLinkageFromMatrix(dist.get(), sizes, reps, numPoints, m, kWardL, tree.get(), s));
  std::vector<double> host((size_t)(m - 1) * 4);
  CUHC_TRY(st, cudaMemcpyAsync(host.data(), tree.get(), tree.bytes(), cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaStreamSynchronize(s));
  if (!st.ok())
    return st.code;
  // Tree ids -> representative points: a new cluster is represented by the
  // representative of its first child.
  std::vector<int> repOfStep(m - 1, -1);
  auto repOf = [&](double id, int step) {
    const long long c = id >= 0 && id < (double)numPoints + step ? (long long)id : -1;
    return c < 0 ? -1 : c < numPoints ? (int)c : repOfStep[c - numPoints];
  };
  u.resize(m - 1);
  v.resize(m - 1);
  h.resize(m - 1);
  for (int step = 0; step < m - 1; ++step) {
    const double *row = &host[(size_t)step * 4];
    u[step] = repOf(row[0], step);
    v[step] = repOf(row[1], step);
    h[step] = (float)row[2];
    repOfStep[step] = u[step];
  }
  return 0;
}

} // namespace cuhc
