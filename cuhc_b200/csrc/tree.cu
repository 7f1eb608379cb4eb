// Edge sorting on the device and merge-tree assembly on the host.
#include "profiling.cuh"
#include "mst.cuh"

#include <algorithm>
#include <cmath>
#include <cub/device/device_radix_sort.cuh>
#include <numeric>

namespace cuhc {
namespace {

__global__ void edgeKeys(const int *__restrict__ u, const float *__restrict__ w,
                         const int *__restrict__ perm, unsigned long long *__restrict__ keys,
                         int m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m)
    return;
  const int e = perm[i];
  // Edge weights are >= 0 (clamped keys), so their bits order like floats.
  keys[i] = ((unsigned long long)floatBits(w[e]) << 32) | (uint32_t)u[e];
}

__global__ void gatherEdges(const int *__restrict__ perm, const int *__restrict__ u,
                            const int *__restrict__ v, const float *__restrict__ w,
                            int *__restrict__ uo, int *__restrict__ vo, float *__restrict__ wo,
                            int m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m)
    return;
  const int e = perm[i];
  uo[i] = u[e];
  vo[i] = v[e];
  wo[i] = w[e];
}

__global__ void iota(int *a, int m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m)
    a[i] = i;
}

} // namespace

namespace {

// Sorts the edges on the device into uo, vo, wo (device buffers of m).
int sortEdgesOnDevice(DeviceEdges &edges, int m, cudaStream_t s, DeviceBuffer<int> &uo,
                      DeviceBuffer<int> &vo, DeviceBuffer<float> &wo) {
  StatusChain st;
  DeviceBuffer<int> perm, perm2, vKeysOut;
  DeviceBuffer<unsigned long long> keys, keysOut;
  CUHC_TRY(st, perm.allocate(m, s));
  CUHC_TRY(st, perm2.allocate(m, s));
  CUHC_TRY(st, vKeysOut.allocate(m, s));
  CUHC_TRY(st, keys.allocate(m, s));
  CUHC_TRY(st, keysOut.allocate(m, s));
  if (!st.ok())
    return st.code;
  const int blocks = (m + 255) / 256;
  iota<<<blocks, 256, 0, s>>>(perm.get(), m); noteLaunch();
  // Least significant key first: stable sort by v, then by (weight, u).
  size_t t1 = 0, t2 = 0;
  CUHC_TRY(st, cub::DeviceRadixSort::SortPairs(nullptr, t1, (const int *)edges.v.get(),
                                               vKeysOut.get(), perm.get(), perm2.get(), m, 0, 32,
                                               s));
  CUHC_TRY(st, cub::DeviceRadixSort::SortPairs(nullptr, t2, keys.get(), keysOut.get(),
                                               perm2.get(), perm.get(), m, 0, 64, s));
  DeviceBuffer<unsigned char> temp;
  CUHC_TRY(st, temp.allocate(std::max(t1, t2), s));
  CUHC_TRY(st, cub::DeviceRadixSort::SortPairs(temp.get(), t1, (const int *)edges.v.get(),
                                               vKeysOut.get(), perm.get(), perm2.get(), m, 0, 32,
                                               s));
  edgeKeys<<<blocks, 256, 0, s>>>(edges.u.get(), edges.w.get(), perm2.get(), keys.get(), m); noteLaunch();
  CUHC_TRY(st, cub::DeviceRadixSort::SortPairs(temp.get(), t2, keys.get(), keysOut.get(),
                                               perm2.get(), perm.get(), m, 0, 64, s));
  gatherEdges<<<blocks, 256, 0, s>>>(perm.get(), edges.u.get(), edges.v.get(), edges.w.get(),
                                     uo.get(), vo.get(), wo.get(), m); noteLaunch();
  CUHC_TRY(st, cudaGetLastError());
  return st.code;
}

// Page-locked host buffers of the calling thread, grown on demand.
struct PinnedEdgeBuffers {
  void *data = nullptr;
  size_t capacity = 0; // edges
  ~PinnedEdgeBuffers() {
    if (data)
      cudaFreeHost(data);
  }
  int reserve(size_t m) {
    if (m <= capacity)
      return 0;
    if (data)
      cudaFreeHost(data);
    data = nullptr;
    capacity = 0;
    const cudaError_t e = cudaHostAlloc(&data, m * (2 * sizeof(int) + sizeof(float)),
                                        cudaHostAllocDefault);
    if (e != cudaSuccess) {
      data = nullptr;
      return (int)e;
    }
    capacity = m;
    return 0;
  }
};

} // namespace

int sortEdgesToHost(DeviceEdges &edges, int m, cudaStream_t s, std::vector<int> &u,
                    std::vector<int> &v, std::vector<float> &w) {
  u.resize(m);
  v.resize(m);
  w.resize(m);
  if (m == 0)
    return 0;
  StatusChain st;
  DeviceBuffer<int> uo, vo;
  DeviceBuffer<float> wo;
  CUHC_TRY(st, uo.allocate(m, s));
  CUHC_TRY(st, vo.allocate(m, s));
  CUHC_TRY(st, wo.allocate(m, s));
  CUHC_TRY(st, sortEdgesOnDevice(edges, m, s, uo, vo, wo));
  CUHC_TRY(st, cudaMemcpyAsync(u.data(), uo.get(), m * sizeof(int), cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaMemcpyAsync(v.data(), vo.get(), m * sizeof(int), cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaMemcpyAsync(w.data(), wo.get(), m * sizeof(float), cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaStreamSynchronize(s));
  return st.code;
}

namespace {

// Instance of each sorted edge (the last i with offsets[i] <= u) and its
// endpoints in the instance's local ids; counts[i] += 1.
__global__ void localiseEdges(const long long *__restrict__ offsets, int count,
                              int *__restrict__ u, int *__restrict__ v,
                              int *__restrict__ instance, int *__restrict__ counts, int m) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m)
    return;
  int lo = 0, hi = count; // offsets[lo] <= u[e] < offsets[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) / 2;
    if (offsets[mid] <= u[e])
      lo = mid;
    else
      hi = mid;
  }
  instance[e] = lo;
  u[e] -= (int)offsets[lo];
  v[e] -= (int)offsets[lo];
  atomicAdd(&counts[lo], 1);
}

PinnedEdgeBuffers &threadPinnedEdges() {
  static thread_local PinnedEdgeBuffers pinned;
  return pinned;
}

} // namespace

int sortBatchEdgesToPinned(DeviceEdges &edges, int m, const std::vector<long long> &offsets,
                           cudaStream_t s, HostEdges &out, std::vector<int> &counts) {
  out = HostEdges{};
  const int count = (int)offsets.size() - 1;
  counts.assign(count, 0);
  if (m == 0)
    return 0;
  PinnedEdgeBuffers &pinned = threadPinnedEdges();
  StatusChain st;
  CUHC_TRY(st, pinned.reserve((size_t)m));
  if (!st.ok())
    return st.code;
  int *hu = static_cast<int *>(pinned.data);
  int *hv = hu + pinned.capacity;
  float *hw = reinterpret_cast<float *>(hv + pinned.capacity);
  DeviceBuffer<int> uo, vo, instance, instanceOut, perm, permOut, ug, vg, devCounts;
  DeviceBuffer<float> wo, wg;
  DeviceBuffer<long long> devOffsets;
  CUHC_TRY(st, uo.allocate(m, s));
  CUHC_TRY(st, vo.allocate(m, s));
  CUHC_TRY(st, wo.allocate(m, s));
  CUHC_TRY(st, instance.allocate(m, s));
  CUHC_TRY(st, instanceOut.allocate(m, s));
  CUHC_TRY(st, perm.allocate(m, s));
  CUHC_TRY(st, permOut.allocate(m, s));
  CUHC_TRY(st, ug.allocate(m, s));
  CUHC_TRY(st, vg.allocate(m, s));
  CUHC_TRY(st, wg.allocate(m, s));
  CUHC_TRY(st, devCounts.allocate(count, s));
  CUHC_TRY(st, devOffsets.allocate(count + 1, s));
  if (!st.ok())
    return st.code;
  CUHC_TRY(st, cudaMemcpyAsync(devOffsets.get(), offsets.data(), (count + 1) * sizeof(long long),
                               cudaMemcpyHostToDevice, s));
  CUHC_TRY(st, cudaMemsetAsync(devCounts.get(), 0, count * sizeof(int), s));
  CUHC_TRY(st, sortEdgesOnDevice(edges, m, s, uo, vo, wo));
  const int blocks = (m + 255) / 256;
  localiseEdges<<<blocks, 256, 0, s>>>(devOffsets.get(), count, uo.get(), vo.get(),
                                       instance.get(), devCounts.get(), m);
  noteLaunch();
  iota<<<blocks, 256, 0, s>>>(perm.get(), m); noteLaunch();
  // Stable by instance: each instance's edges keep their (w, u, v) order.
  int bits = 1;
  while ((1 << bits) < count)
    ++bits;
  size_t tempBytes = 0;
  CUHC_TRY(st, cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, instance.get(),
                                               instanceOut.get(), perm.get(), permOut.get(), m,
                                               0, bits, s));
  DeviceBuffer<unsigned char> temp;
  CUHC_TRY(st, temp.allocate(std::max<size_t>(tempBytes, 1), s));
  CUHC_TRY(st, cub::DeviceRadixSort::SortPairs(temp.get(), tempBytes, instance.get(),
                                               instanceOut.get(), perm.get(), permOut.get(), m,
                                               0, bits, s));
  gatherEdges<<<blocks, 256, 0, s>>>(permOut.get(), uo.get(), vo.get(), wo.get(), ug.get(),
                                     vg.get(), wg.get(), m);
  noteLaunch();
  CUHC_TRY(st, cudaGetLastError());
  CUHC_TRY(st, cudaMemcpyAsync(hu, ug.get(), m * sizeof(int), cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaMemcpyAsync(hv, vg.get(), m * sizeof(int), cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaMemcpyAsync(hw, wg.get(), m * sizeof(float), cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaMemcpyAsync(counts.data(), devCounts.get(), count * sizeof(int),
                               cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaStreamSynchronize(s));
  if (st.ok())
    out = HostEdges{hu, hv, hw, m};
  return st.code;
}

int sortEdgesToPinned(DeviceEdges &edges, int m, cudaStream_t s, HostEdges &out) {
  PinnedEdgeBuffers &pinned = threadPinnedEdges();
  out = HostEdges{};
  if (m == 0)
    return 0;
  StatusChain st;
  CUHC_TRY(st, pinned.reserve((size_t)m));
  if (!st.ok())
    return st.code;
  int *hu = static_cast<int *>(pinned.data);
  int *hv = hu + pinned.capacity;
  float *hw = reinterpret_cast<float *>(hv + pinned.capacity);
  DeviceBuffer<int> uo, vo;
  DeviceBuffer<float> wo;
  CUHC_TRY(st, uo.allocate(m, s));
  CUHC_TRY(st, vo.allocate(m, s));
  CUHC_TRY(st, wo.allocate(m, s));
  CUHC_TRY(st, sortEdgesOnDevice(edges, m, s, uo, vo, wo));
  CUHC_TRY(st, cudaMemcpyAsync(hu, uo.get(), m * sizeof(int), cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaMemcpyAsync(hv, vo.get(), m * sizeof(int), cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaMemcpyAsync(hw, wo.get(), m * sizeof(float), cudaMemcpyDeviceToHost, s));
  CUHC_TRY(st, cudaStreamSynchronize(s));
  if (st.ok())
    out = HostEdges{hu, hv, hw, m};
  return st.code;
}

namespace {
inline int findRoot(std::vector<int> &parent, int x) {
  while (parent[x] != x) {
    parent[x] = parent[parent[x]];
    x = parent[x];
  }
  return x;
}
} // namespace

void treeFromOrderedMerges(const std::vector<int> &u, const std::vector<int> &v,
                           const std::vector<float> &w, int n, double *Z) {
  treeFromOrderedMerges(u.data(), v.data(), w.data(), n, Z);
}

// Union-find over the merges in order. A node's parent, size and cluster id
// share one 16-byte record (one cache line per touch), and the records of
// the endpoints kPrefetch merges ahead are prefetched: the loop is bound by
// the latency of those random first touches, not by its arithmetic.
void treeFromOrderedMerges(const int *u, const int *v, const float *w, int n, double *Z) {
  struct Node {
    int parent, size, id, unused;
  };
  constexpr int kPrefetch = 16;
  // Reused by the thread's later calls: a fresh 16-byte record per point
  // would cost a page fault per 256 points on every call.
  static thread_local std::vector<Node> node;
  if (node.size() < (size_t)n)
    node.resize(n);
  for (int i = 0; i < n; ++i)
    node[i] = {i, 1, i, 0};
  auto find = [](int x) {
    while (node[x].parent != x) {
      node[x].parent = node[node[x].parent].parent;
      x = node[x].parent;
    }
    return x;
  };
  for (int s = 0; s < n - 1; ++s) {
    if (s + kPrefetch < n - 1) {
      __builtin_prefetch(&node[u[s + kPrefetch]], 1);
      __builtin_prefetch(&node[v[s + kPrefetch]], 1);
    }
    int ru = find(u[s]), rv = find(v[s]);
    const int a = node[ru].id, b = node[rv].id;
    const int merged = node[ru].size + node[rv].size;
    double *row = Z + (size_t)s * 4;
    row[0] = std::min(a, b);
    row[1] = std::max(a, b);
    row[2] = w[s];
    row[3] = merged;
    if (node[ru].size < node[rv].size)
      std::swap(ru, rv);
    node[rv].parent = ru;
    node[ru].size = merged;
    node[ru].id = n + s;
  }
}

bool mergesFormTree(const std::vector<int> &u, const std::vector<int> &v,
                    const std::vector<float> &w, int n) {
  if ((int)u.size() != n - 1)
    return false;
  std::vector<int> parent(n);
  std::iota(parent.begin(), parent.end(), 0);
  for (int s = 0; s < n - 1; ++s) {
    if (!std::isfinite(w[s]) || u[s] < 0 || u[s] >= n || v[s] < 0 || v[s] >= n)
      return false;
    const int ru = findRoot(parent, u[s]), rv = findRoot(parent, v[s]);
    if (ru == rv)
      return false;
    parent[rv] = ru;
  }
  return true;
}

} // namespace cuhc
