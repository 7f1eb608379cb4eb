// The C ABI of libcuhc.so (declared in include/cuhc.h).
//
// The first eight functions are the reference's ctypes boundary
// (capi.cu:133-366 of shangar21/cuhc) with the same names, signatures,
// argument meaning, id tables, validation order and status codes, so the
// reference's Python layer can load this library unchanged. Host pointers in,
// host results out; device memory comes from the stream-ordered pool.
//
// The other functions are additions with no counterpart in the reference:
// device-pointer variants (inputs already in HBM, for callers that keep data
// on the GPU) and extended pass statistics.
#include <algorithm>
#include <atomic>
#include <map>
#include <cmath>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include "profiling.cuh"
#include "mst.cuh"
#include "metrics.cuh"
#include "pairwise.cuh"
#include "rnn.cuh"
#include "screen.cuh"

namespace cuhc {

// Linkage ids (reference linkage.cuh:31) and algorithm ids (capi.cu:33-38).
enum LinkageId : int { kSingle = 0, kComplete = 1, kAverage = 2, kWard = 3 };
enum AlgorithmId : int { kDense = 0, kMst = 1, kNnChain = 2, kRnn = 3 };
// Pruning modes of cuhc_set_pruning (reference spatial.cuh:354).
enum PruneMode : int { kPruneAuto = 0, kPruneAlways = 1, kPruneNever = 2 };
// Core-distance methods (reference hdbscan.cuh:324).
enum CoreMethod : int { kCoreAuto = 0, kCoreFused = 1, kCoreRadix = 2 };
constexpr int kMaxFusedK = 64;     // reference hdbscan.cuh:112
constexpr int kMaxPruneFeatures = 256;
// Largest k whose per-row lists fit in shared memory (128 rows x k floats);
// larger k uses radix select.
constexpr int kMaxListK = 256;
// Largest k whose lists are kept for the Borůvka seeds (values and positions
// in shared memory).
constexpr int kMaxKeptListK = 64;

std::atomic<int> gPruneMode{kPruneAuto};
std::mutex gStatsMutex;
PassStats gStats;

int currentPruneMode() { return gPruneMode.load(); }

std::atomic<int> gScreenMode{0};
// Set by the batched path's autotuner for the duration of one call.
thread_local int tScreenOverride = -1;
int currentScreenMode() { return tScreenOverride >= 0 ? tScreenOverride : gScreenMode.load(); }
thread_local ScreenShape tScreenShape;
std::atomic<int> gLastShapeStages{0}, gLastShapeLead{0};
ScreenShape currentScreenShape() { return tScreenShape; }
void setScreenShape(ScreenShape shape) {
  tScreenShape = shape;
  if (shape.stages > 0) {
    gLastShapeStages.store(shape.stages);
    gLastShapeLead.store(shape.lead);
  }
}

int pairwiseIntoMatrix(const float *points, int n, int d, int metricId, float p, float *out,
                       cudaStream_t s) {
  return withMetric(metricId, p, [&](auto m) {
    return pairwiseDistances(points, n, nullptr, n, d, m, out, s);
  });
}

void addStats(const PassStats &s) {
  std::lock_guard<std::mutex> lock(gStatsMutex);
  gStats.tilesComputed += s.tilesComputed;
  gStats.tilesTotal += s.tilesTotal;
  gStats.passes += s.passes;
  gStats.rounds += s.rounds;
}

// Whether a call builds the k-d order and prunes with boxes. Results never
// depend on it. "auto" prunes whenever the metric has a box bound: the GPU
// k-d build costs about one pass of a small input, and the traversal is
// nearly free when boxes separate nothing.
template <class Metric> bool shouldPrune(int n, int d) {
  const int mode = gPruneMode.load();
  return Metric::kBoxBound && mode != kPruneNever && numTilesFor(n) >= 2 && d <= kMaxPruneFeatures;
}

// One stream per call, and a pool that keeps its memory between calls.
struct CallContext {
  cudaStream_t stream = nullptr;
  int status = 0;
  CallContext() {
    static std::once_flag once;
    std::call_once(once, [] {
      int device = 0;
      cudaGetDevice(&device);
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        unsigned long long threshold = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
      }
    });
    status = (int)cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  }
  ~CallContext() {
    if (stream) {
      cudaStreamSynchronize(stream);
      cudaStreamDestroy(stream);
    }
  }
};

__global__ void scatterByOrder(const float *__restrict__ byPosition, const int *__restrict__ order,
                               float *__restrict__ byOriginal, int n) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n && order[p] >= 0) // padding slots of a batch hold no point
    byOriginal[order[p]] = byPosition[p];
}

// Single linkage by Borůvka on device points; tree to the host.
template <class Metric>
int singleLinkageMst(const float *devPoints, int n, int d, const Metric &m, double *hostTree,
                     cudaStream_t s) {
  StatusChain st;
  SpatialIndex index;
  const bool prune = shouldPrune<Metric>(n, d);
  CUHC_TRY(st, index.build(devPoints, n, d, prune, s));
  DeviceEdges edges;
  PassStats stats;
  CUHC_TRY(st, (boruvkaMst<Metric, PlainWeight>(index, m, PlainWeight{}, prune, edges, &stats, s)));
  HostEdges sorted;
  CUHC_TRY(st, sortEdgesToPinned(edges, edges.count, s, sorted));
  if (st.ok() && sorted.count != n - 1)
    st(kErrorDisconnected);
  if (st.ok())
    treeFromOrderedMerges(sorted.u, sorted.v, sorted.w, n, hostTree);
  addStats(stats);
  return st.code;
}

template <class Metric>
int hdbscanTree(const float *devPoints, int n, int d, const Metric &m, int minSamples, float alpha,
                int coreMethod, double *hostTree, float *hostCore, cudaStream_t s) {
  StatusChain st;
  SpatialIndex index;
  const bool prune = shouldPrune<Metric>(n, d);
  CUHC_TRY(st, index.build(devPoints, n, d, prune, s));
  DeviceBuffer<float> core, coreOrig;
  CUHC_TRY(st, core.allocate(paddedToTiles(n), s));
  PassStats stats;
  // The k-NN pass also keeps every point's list (positions, boundary tie),
  // which lets the Borůvka rounds settle most rows without a search; with
  // alpha 1 only (a list edge's weight then needs no distance) and lists
  // that fit shared memory twice over.
  const bool radix = coreMethod == kCoreRadix || minSamples > kMaxListK;
  const bool keepLists = !radix && alpha == 1.0f && minSamples <= kMaxKeptListK && n > 1;
  DeviceBuffer<int> knnPos, knnTie;
  if (keepLists) {
    CUHC_TRY(st, knnPos.allocate((size_t)n * minSamples, s));
    CUHC_TRY(st, knnTie.allocate(n, s));
  }
  // Radix select when asked for, or when the per-row lists would not fit
  // shared memory (the reference's Auto picks radix above k = 64).
  if (radix)
    CUHC_TRY(st, coreDistancesRadix<Metric>(index, m, minSamples, core.get(), s));
  else
    CUHC_TRY(st, coreDistances<Metric>(index, m, minSamples, prune, core.get(), &stats, s,
                                       nullptr, knnPos.get(), knnTie.get()));
  CUHC_TRY(st, index.updateMinValues(core.get()));
  DeviceEdges edges;
  MutualReachWeight weight;
  weight.value = core.get();
  weight.alpha = alpha;
  KnnLists lists;
  lists.pos = knnPos.get();
  lists.tie = knnTie.get();
  lists.k = minSamples;
  if (n > 1)
    CUHC_TRY(st, (boruvkaMst<Metric, MutualReachWeight>(index, m, weight, prune, edges, &stats, s,
                                                        nullptr, keepLists ? &lists : nullptr)));
  if (hostCore && st.ok()) {
    CUHC_TRY(st, coreOrig.allocate(n, s));
    scatterByOrder<<<(n + 255) / 256, 256, 0, s>>>(core.get(), index.order.get(), coreOrig.get(),
                                                   n); noteLaunch();
    CUHC_TRY(st, cudaGetLastError());
    CUHC_TRY(st, cudaMemcpyAsync(hostCore, coreOrig.get(), n * sizeof(float),
                                 cudaMemcpyDeviceToHost, s));
  }
  if (n > 1) {
    HostEdges sorted;
    CUHC_TRY(st, sortEdgesToPinned(edges, edges.count, s, sorted));
    if (st.ok() && sorted.count != n - 1)
      st(kErrorDisconnected);
    if (st.ok())
      treeFromOrderedMerges(sorted.u, sorted.v, sorted.w, n, hostTree);
  }
  CUHC_TRY(st, cudaStreamSynchronize(s));
  addStats(stats);
  return st.code;
}

// ---- batched trees (many instances, one solve per call) ----

// Autotuner of the batched path: for (metric, d) the faster of the screened
// and the plain k-NN kernel, timed once per process on the first 2 x SMs row
// tiles of a batch (after one warm-up launch of each). The choice changes
// time only, never a result. Returns the screen mode to use (1 on, 2 off).
std::mutex gTuneMutex;
std::map<std::pair<int, int>, int> gTuned;

template <class Metric>
int tuneScreen(SpatialIndex &index, const Metric &m, int metricId, int k, float *scratch,
               cudaStream_t s) {
  if (gScreenMode.load() != 0)
    return gScreenMode.load();
  if (!screenable<Metric>(index, k))
    return 2;
  const std::pair<int, int> key(metricId, index.d);
  {
    std::lock_guard<std::mutex> lock(gTuneMutex);
    const auto it = gTuned.find(key);
    if (it != gTuned.end())
      return it->second;
  }
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int sample = 2 * sms;
  float best[2] = {INFINITY, INFINITY};
  for (int rep = 0; rep < 3; ++rep)
    for (int v = 0; v < 2; ++v) {
      const float ms = timeKnnSample(index, m, k, v == 0, sample, scratch, s);
      if (rep > 0)
        best[v] = std::min(best[v], ms);
    }
  const int mode = best[0] <= best[1] ? 1 : 2;
  std::lock_guard<std::mutex> lock(gTuneMutex);
  gTuned[key] = mode;
  return mode;
}

struct ScreenOverride {
  explicit ScreenOverride(int mode) { tScreenOverride = mode; }
  ~ScreenOverride() { tScreenOverride = -1; }
};

template <class Metric>
int batchTrees(const float *devPoints, const std::vector<int> &sizes,
               const std::vector<long long> &offsets, int d, const Metric &m, int metricId,
               const int *minSamples, double *hostTrees, float *hostCore, cudaStream_t s) {
  StatusChain st;
  SpatialIndex index;
  CUHC_TRY(st, index.buildBatch(devPoints, sizes, d, s));
  if (!st.ok())
    return st.code;
  const int count = (int)sizes.size(), positions = index.n;
  int maxK = 0;
  std::vector<int> hostRank(positions, 0);
  for (int i = 0; i < count; ++i) {
    maxK = std::max(maxK, minSamples[i]);
    const int base = index.instanceFirstTile[i] * kTile;
    std::fill(hostRank.begin() + base, hostRank.begin() + base + sizes[i], minSamples[i]);
  }
  DeviceBuffer<float> core;
  DeviceBuffer<int> rank;
  CUHC_TRY(st, core.allocate(paddedToTiles(positions), s));
  CUHC_TRY(st, rank.allocate(positions, s));
  CUHC_TRY(st, cudaMemsetAsync(core.get(), 0, core.bytes(), s));
  CUHC_TRY(st, cudaMemcpyAsync(rank.get(), hostRank.data(), positions * sizeof(int),
                               cudaMemcpyHostToDevice, s));
  CUHC_TRY(st, cudaStreamSynchronize(s));
  if (!st.ok())
    return st.code;
  ScreenOverride screen(tuneScreen(index, m, metricId, std::max(maxK, 1), core.get(), s));
  CUHC_TRY(st, cudaMemsetAsync(core.get(), 0, core.bytes(), s));
  PassStats stats;
  // Mutual reachability with core 0 is the plain distance (keys clamp at 0),
  // so single-linkage instances (rank 0) share the solve with HDBSCAN ones.
  if (maxK > 0)
    CUHC_TRY(st, coreDistances<Metric>(index, m, maxK, true, core.get(), &stats, s, rank.get()));
  CUHC_TRY(st, index.updateMinValues(core.get()));
  MutualReachWeight weight;
  weight.value = core.get();
  weight.alpha = 1.0f;
  DeviceEdges edges;
  CUHC_TRY(st, (boruvkaMst<Metric, MutualReachWeight>(index, m, weight, true, edges, &stats, s)));
  // Edges sorted by (instance, w, u, v) on the device, in local ids: instance
  // i's n_i - 1 edges at slots offsets[i] - i ...; then every instance's tree
  // on the host threads.
  HostEdges sorted;
  std::vector<int> edgeCounts;
  CUHC_TRY(st, sortBatchEdgesToPinned(edges, edges.count, offsets, s, sorted, edgeCounts));
  if (st.ok() && (long long)sorted.count != offsets[count] - count)
    st(kErrorDisconnected);
  for (int i = 0; st.ok() && i < count; ++i)
    if (edgeCounts[i] != sizes[i] - 1)
      st(kErrorDisconnected);
  if (st.ok()) {
    std::atomic<int> next{0};
    auto worker = [&]() {
      for (int i = next++; i < count; i = next++) {
        const long long first = offsets[i] - i;
        treeFromOrderedMerges(sorted.u + first, sorted.v + first, sorted.w + first, sizes[i],
                              hostTrees + first * 4);
      }
    };
    if (st.ok()) {
      const int threads =
          (int)std::max(1u, std::min(std::thread::hardware_concurrency(), (unsigned)count));
      std::vector<std::thread> pool;
      for (int t = 1; t < threads; ++t)
        pool.emplace_back(worker);
      worker();
      for (auto &th : pool)
        th.join();
    }
  }
  if (hostCore && st.ok()) {
    DeviceBuffer<float> coreOrig;
    CUHC_TRY(st, coreOrig.allocate(index.numPoints, s));
    scatterByOrder<<<(positions + 255) / 256, 256, 0, s>>>(core.get(), index.order.get(),
                                                           coreOrig.get(), positions);
    noteLaunch();
    CUHC_TRY(st, cudaGetLastError());
    CUHC_TRY(st, cudaMemcpyAsync(hostCore, coreOrig.get(), index.numPoints * sizeof(float),
                                 cudaMemcpyDeviceToHost, s));
  }
  CUHC_TRY(st, cudaStreamSynchronize(s));
  addStats(stats);
  return st.code;
}

int validateLinkage(int n, int d, int metricId, int linkageId, int algorithmId) {
  if (n <= 0 || d <= 0)
    return kErrorInvalidShape;
  if (linkageId < kSingle || linkageId > kWard)
    return kErrorInvalidLinkage;
  const bool valid = algorithmId == kDense || (algorithmId == kMst && linkageId == kSingle) ||
                     ((algorithmId == kNnChain || algorithmId == kRnn) && linkageId == kWard &&
                      metricId == kEuclidean);
  if (!valid)
    return kErrorInvalidAlgorithm;
  if (metricId < kEuclidean || metricId > kCosine)
    return kErrorInvalidMetric;
  return 0;
}

int linkageOnDevice(const float *devPoints, int n, int d, int metricId, float p, int linkageId,
                    int algorithmId, double *hostTree, cudaStream_t s) {
  if (algorithmId == kMst)
    return withMetric(metricId, p, [&](auto m) {
      return singleLinkageMst(devPoints, n, d, m, hostTree, s);
    });
  if (algorithmId == kRnn) {
    RnnOptions options;
    PassStats stats;
    const int status = rnnWard(devPoints, n, d, options, hostTree, &stats, s);
    addStats(stats);
    return status;
  }
  if (algorithmId == kNnChain)
    return nnChainWard(devPoints, n, d, hostTree, s);
  return denseLinkage(devPoints, n, d, metricId, p, linkageId, hostTree, s);
}

int validateHdbscan(int n, int d, int minSamples, int coreMethod) {
  if (n <= 0 || d <= 0 || minSamples < 1 || minSamples > n)
    return kErrorInvalidShape;
  if (coreMethod < 0 || coreMethod > 2 || (coreMethod == kCoreFused && minSamples > kMaxFusedK))
    return kErrorInvalidAlgorithm;
  return 0;
}

} // namespace cuhc

using namespace cuhc;

extern "C" {

// The pipeline shape (ring slots, copy lead) the shape tuner chose for the
// latest screened k-NN pass of any thread (0, 0 before any). Diagnostic.
int cuhc_screen_shape(int *stages, int *lead) {
  if (!stages || !lead)
    return cuhc::kErrorInvalidShape;
  *stages = cuhc::gLastShapeStages.load();
  *lead = cuhc::gLastShapeLead.load();
  return 0;
}

int cuhc_pairwise_distances(const float *hostA, int nA, const float *hostB, int nB, int d,
                            int metricId, float p, float *hostOut) {
  if (nA <= 0 || nB <= 0 || d <= 0)
    return kErrorInvalidShape;
  if (metricId < kEuclidean || metricId > kCosine)
    return kErrorInvalidMetric;
  CallContext ctx;
  StatusChain st;
  st(ctx.status);
  cudaStream_t s = ctx.stream;
  DeviceBuffer<float> A, B, out;
  CUHC_TRY(st, A.allocate((size_t)nA * d, s));
  CUHC_TRY(st, out.allocate((size_t)nA * nB, s));
  CUHC_TRY(st, cudaMemcpyAsync(A.get(), hostA, A.bytes(), cudaMemcpyHostToDevice, s));
  if (hostB) {
    CUHC_TRY(st, B.allocate((size_t)nB * d, s));
    CUHC_TRY(st, cudaMemcpyAsync(B.get(), hostB, B.bytes(), cudaMemcpyHostToDevice, s));
  }
  if (st.ok())
    st(withMetric(metricId, p, [&](auto m) {
      return pairwiseDistances(A.get(), nA, hostB ? B.get() : nullptr, nB, d, m, out.get(), s);
    }));
  CUHC_TRY(st, cudaMemcpyAsync(hostOut, out.get(), out.bytes(), cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaStreamSynchronize(s));
  return st.code;
}

int cuhc_linkage(const float *hostPoints, int n, int d, int metricId, float p, int linkageId,
                 int algorithmId, double *hostTree) {
  const int invalid = validateLinkage(n, d, metricId, linkageId, algorithmId);
  if (invalid)
    return invalid;
  if (n == 1)
    return 0;
  CallContext ctx;
  StatusChain st;
  st(ctx.status);
  DeviceBuffer<float> points;
  CUHC_TRY(st, points.allocate((size_t)n * d, ctx.stream));
  CUHC_TRY(st, cudaMemcpyAsync(points.get(), hostPoints, points.bytes(), cudaMemcpyHostToDevice,
                               ctx.stream));
  CUHC_TRY(st, linkageOnDevice(points.get(), n, d, metricId, p, linkageId, algorithmId, hostTree,
                               ctx.stream));
  return st.code;
}

int cuhc_ward_rnn_with_options(const float *hostPoints, int n, int d, float minProgress,
                               int denseBelow, int allowDense, double *hostTree) {
  if (n <= 0 || d <= 0)
    return kErrorInvalidShape;
  if (n == 1)
    return 0;
  CallContext ctx;
  StatusChain st;
  st(ctx.status);
  DeviceBuffer<float> points;
  CUHC_TRY(st, points.allocate((size_t)n * d, ctx.stream));
  CUHC_TRY(st, cudaMemcpyAsync(points.get(), hostPoints, points.bytes(), cudaMemcpyHostToDevice,
                               ctx.stream));
  RnnOptions options;
  options.minProgress = minProgress;
  options.denseBelow = denseBelow;
  options.allowDense = allowDense != 0;
  PassStats stats;
  CUHC_TRY(st, rnnWard(points.get(), n, d, options, hostTree, &stats, ctx.stream));
  addStats(stats);
  return st.code;
}

int cuhc_hdbscan_tree(const float *hostPoints, int n, int d, int metricId, float p,
                      int minSamples, float alpha, int coreMethod, double *hostTree,
                      float *hostCore) {
  const int invalid = validateHdbscan(n, d, minSamples, coreMethod);
  if (invalid)
    return invalid;
  if (metricId < kEuclidean || metricId > kCosine)
    return kErrorInvalidMetric;
  CallContext ctx;
  StatusChain st;
  st(ctx.status);
  DeviceBuffer<float> points;
  CUHC_TRY(st, points.allocate((size_t)n * d, ctx.stream));
  CUHC_TRY(st, cudaMemcpyAsync(points.get(), hostPoints, points.bytes(), cudaMemcpyHostToDevice,
                               ctx.stream));
  if (st.ok())
    st(withMetric(metricId, p, [&](auto m) {
      return hdbscanTree(points.get(), n, d, m, minSamples, alpha, coreMethod, hostTree, hostCore,
                         ctx.stream);
    }));
  return st.code;
}

long long cuhc_condense_tree(const double *tree, long long n, long long minClusterSize,
                             long long capacity, long long *parent, long long *child,
                             double *lambda, long long *size) {
  return condenseTree(tree, n, minClusterSize, capacity, parent, child, lambda, size);
}

namespace {
// Checks a batch description; sizes receives the instances' row counts.
int validateBatch(const long long *offsets, int count, int d, int metricId,
                  const int *minSamples, std::vector<int> &sizes) {
  if (count < 1 || d < 1 || !offsets || !minSamples || offsets[0] != 0)
    return kErrorInvalidShape;
  sizes.assign(count, 0);
  long long positions = 0;
  for (int i = 0; i < count; ++i) {
    const long long n = offsets[i + 1] - offsets[i];
    if (n < 1 || minSamples[i] < 0 || minSamples[i] > n)
      return kErrorInvalidShape;
    if (n > (1LL << 30))
      return kErrorTooLarge;
    sizes[i] = (int)n;
    positions += (long long)numTilesFor((int)n) * kTile;
  }
  if (positions > (1LL << 30) || offsets[count] * (long long)d > (1LL << 40))
    return kErrorTooLarge;
  for (int i = 0; i < count; ++i)
    if (minSamples[i] > kMaxListK)
      return kErrorTooLarge;
  if (metricId < kEuclidean || metricId > kCosine)
    return kErrorInvalidMetric;
  return 0;
}
} // namespace

int cuhc_trees_batched(const float *hostPoints, const long long *offsets, int count, int d,
                       int metricId, float p, const int *minSamples, double *trees,
                       float *core) {
  std::vector<int> sizes;
  const int invalid = validateBatch(offsets, count, d, metricId, minSamples, sizes);
  if (invalid)
    return invalid;
  std::vector<long long> off(offsets, offsets + count + 1);
  CallContext ctx;
  StatusChain st;
  st(ctx.status);
  DeviceBuffer<float> points;
  CUHC_TRY(st, points.allocate((size_t)offsets[count] * d, ctx.stream));
  CUHC_TRY(st, cudaMemcpyAsync(points.get(), hostPoints, points.bytes(), cudaMemcpyHostToDevice,
                               ctx.stream));
  if (st.ok())
    st(withMetric(metricId, p, [&](auto m) {
      return batchTrees(points.get(), sizes, off, d, m, metricId, minSamples, trees, core,
                        ctx.stream);
    }));
  return st.code;
}

int cuhc_trees_batched_device(const float *devicePoints, const long long *offsets, int count,
                              int d, int metricId, float p, const int *minSamples, double *trees,
                              float *core) {
  std::vector<int> sizes;
  const int invalid = validateBatch(offsets, count, d, metricId, minSamples, sizes);
  if (invalid)
    return invalid;
  std::vector<long long> off(offsets, offsets + count + 1);
  CallContext ctx;
  StatusChain st;
  st(ctx.status);
  if (st.ok())
    st(withMetric(metricId, p, [&](auto m) {
      return batchTrees(devicePoints, sizes, off, d, m, metricId, minSamples, trees, core,
                        ctx.stream);
    }));
  return st.code;
}

// Training rows for the radius model: runs the single-linkage Borůvka rounds
// of points (HOST, n x 16) exactly and keeps up to maxRowsPerRound random
// rows per round (seeded) of (19 features, log nearest other-component
// weight). Writes min(rows, capacity) rows; *rows receives the count found.
int cuhc_radius_training_rows(const float *hostPoints, int n, int d, int maxRowsPerRound,
                              unsigned long long seed, float *features, float *targets,
                              long long capacity, long long *rows) {
  if (n < 2 || d != kRadiusDims || maxRowsPerRound < 1 || capacity < 0)
    return kErrorInvalidShape;
  CallContext ctx;
  StatusChain st;
  st(ctx.status);
  DeviceBuffer<float> points;
  CUHC_TRY(st, points.allocate((size_t)n * d, ctx.stream));
  CUHC_TRY(st, cudaMemcpyAsync(points.get(), hostPoints, points.bytes(), cudaMemcpyHostToDevice,
                               ctx.stream));
  RadiusLog log;
  log.maxRowsPerRound = maxRowsPerRound;
  log.seed = seed;
  SpatialIndex index;
  CUHC_TRY(st, index.build(points.get(), n, d, true, ctx.stream));
  DeviceEdges edges;
  PassStats stats;
  EuclideanMetric m;
  CUHC_TRY(st, (boruvkaMst<EuclideanMetric, PlainWeight>(index, m, PlainWeight{}, true, edges,
                                                          &stats, ctx.stream, &log)));
  const long long found = (long long)log.targets.size();
  if (rows)
    *rows = found;
  const long long keep = std::min(found, capacity);
  if (st.ok() && keep > 0) {
    std::copy(log.features.begin(), log.features.begin() + keep * kRadiusFeatures, features);
    std::copy(log.targets.begin(), log.targets.begin() + keep, targets);
  }
  return st.code;
}

int cuhc_set_pruning(int mode) {
  if (mode < kPruneAuto || mode > kPruneNever)
    return kErrorInvalidAlgorithm;
  gPruneMode.store(mode);
  return 0;
}

// Tensor-core screening of the all-pairs passes (an addition): 0 auto (on
// for euclidean / sqeuclidean with d <= 32), 1 on where supported, 2 off.
// Results are identical in every mode; only the time changes.
int cuhc_set_screen(int mode) {
  if (mode < 0 || mode > 2)
    return kErrorInvalidAlgorithm;
  gScreenMode.store(mode);
  return 0;
}

void cuhc_prune_stats(unsigned long long *computed, unsigned long long *total) {
  std::lock_guard<std::mutex> lock(gStatsMutex);
  *computed = gStats.tilesComputed;
  *total = gStats.tilesTotal;
  gStats.tilesComputed = gStats.tilesTotal = 0;
}

const char *cuhc_error_string(int code) {
  switch (code) {
  case kErrorInvalidMetric:
    return "invalid metric id";
  case kErrorInvalidShape:
    return "array dimensions must be positive";
  case kErrorInvalidLinkage:
    return "invalid linkage id";
  case kErrorInvalidAlgorithm:
    return "invalid algorithm id for this linkage";
  case kErrorNonFinite:
    return "distances overflowed float32 or are NaN; rescale the data";
  case kErrorDisconnected:
    return "some points have no finite distance to the others (NaN or infinite values?)";
  case kErrorTimeout:
    return "a device-side wait ran out of its iteration budget";
  case kErrorTooLarge:
    return "input exceeds a documented size limit of this entry point";
  default:
    return cudaGetErrorString((cudaError_t)code);
  }
}

// ---- additions ------------------------------------------------------------

int cuhc_linkage_device(const float *devicePoints, int n, int d, int metricId, float p,
                        int linkageId, int algorithmId, double *hostTree) {
  const int invalid = validateLinkage(n, d, metricId, linkageId, algorithmId);
  if (invalid)
    return invalid;
  if (n == 1)
    return 0;
  CallContext ctx;
  StatusChain st;
  st(ctx.status);
  CUHC_TRY(st, linkageOnDevice(devicePoints, n, d, metricId, p, linkageId, algorithmId, hostTree,
                               ctx.stream));
  return st.code;
}

int cuhc_hdbscan_tree_device(const float *devicePoints, int n, int d, int metricId, float p,
                             int minSamples, float alpha, int coreMethod, double *hostTree,
                             float *hostCore) {
  const int invalid = validateHdbscan(n, d, minSamples, coreMethod);
  if (invalid)
    return invalid;
  if (metricId < kEuclidean || metricId > kCosine)
    return kErrorInvalidMetric;
  CallContext ctx;
  StatusChain st;
  st(ctx.status);
  if (st.ok())
    st(withMetric(metricId, p, [&](auto m) {
      return hdbscanTree(devicePoints, n, d, m, minSamples, alpha, coreMethod, hostTree, hostCore,
                         ctx.stream);
    }));
  return st.code;
}

int cuhc_pairwise_distances_device(const float *devA, int nA, const float *devB, int nB, int d,
                                   int metricId, float p, float *devOut) {
  if (nA <= 0 || nB <= 0 || d <= 0 || (!devB && nB != nA))
    return kErrorInvalidShape;
  if (metricId < kEuclidean || metricId > kCosine)
    return kErrorInvalidMetric;
  CallContext ctx;
  StatusChain st;
  st(ctx.status);
  if (st.ok())
    st(withMetric(metricId, p, [&](auto m) {
      return pairwiseDistances(devA, nA, devB, nB, d, m, devOut, ctx.stream);
    }));
  return st.code;
}

int cuhc_pass_stats(unsigned long long *out, int count) {
  std::lock_guard<std::mutex> lock(gStatsMutex);
  const unsigned long long values[4] = {gStats.tilesComputed, gStats.tilesTotal, gStats.passes,
                                        gStats.rounds};
  for (int i = 0; i < count && i < 4; ++i)
    out[i] = values[i];
  return 0;
}

} // extern "C"
