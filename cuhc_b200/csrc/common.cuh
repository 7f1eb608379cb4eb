// Shared definitions for the cuhc_b200 kernels: status codes, packed argmin
// keys, device buffers from the stream-ordered pool, bounded waits.
#pragma once

#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

namespace cuhc {

// Status codes of the C ABI. Zero is success, positive values are
// cudaError_t, negative values are library errors. The negative codes and
// their meaning are the reference's (capi.cu:26-30, mst.cuh:80-81) so that a
// caller of either library sees the same numbers.
enum Status : int {
  kOk = 0,
  kErrorInvalidMetric = -1,
  kErrorInvalidShape = -2,
  kErrorInvalidLinkage = -3,
  kErrorInvalidAlgorithm = -4,
  kErrorDisconnected = -5,
  kErrorNonFinite = -6,
  // No counterpart in the reference: a bounded device-side wait ran out.
  kErrorTimeout = -7,
  // No counterpart in the reference: a size beyond a documented limit.
  kErrorTooLarge = -8,
};

// First error of a sequence of calls wins.
struct StatusChain {
  int code = 0;
  int operator()(int result) {
    if (code == 0 && result != 0)
      code = result;
    return code;
  }
  bool ok() const { return code == 0; }
};

#define CUHC_TRY(chain, expr)                                                                      \
  do {                                                                                             \
    if ((chain).ok())                                                                              \
      (chain)((int)(expr));                                                                        \
  } while (0)

// ---------------------------------------------------------------------------
// Packed argmin keys.
//
// An edge candidate is (weight, index) packed as (float bits << 32) | index,
// so that comparing keys as unsigned 64-bit integers compares the weight
// first and then the index: non-negative floats order like their bit
// patterns. Weights are clamped at +0 first (cosine rounding can give -1e-8).
// Ties therefore go to the lower index, the reference's rule
// (reductions.cuh:19-21, 64-69). The index is always an ORIGINAL point index,
// whatever order the points are stored in, so ties break the same way as in
// an unpermuted run.
constexpr unsigned long long kEmptyKey = ~0ull;

__host__ __device__ __forceinline__ uint32_t floatBits(float x) {
#ifdef __CUDA_ARCH__
  return __float_as_uint(x);
#else
  uint32_t b;
  memcpy(&b, &x, 4);
  return b;
#endif
}

__host__ __device__ __forceinline__ float bitsFloat(uint32_t b) {
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float x;
  memcpy(&x, &b, 4);
  return x;
#endif
}

__host__ __device__ __forceinline__ unsigned long long packKey(float weight, uint32_t index) {
  const float clamped = weight > 0.0f ? weight : 0.0f;
  return ((unsigned long long)floatBits(clamped) << 32) | index;
}

__host__ __device__ __forceinline__ float keyWeight(unsigned long long key) {
  return bitsFloat((uint32_t)(key >> 32));
}

__host__ __device__ __forceinline__ uint32_t keyIndex(unsigned long long key) {
  return (uint32_t)(key & 0xffffffffull);
}

// Order-preserving map of a float to uint32 (for radix sorts and atomics on
// signed floats): negative values flip all bits, others set the sign bit.
__host__ __device__ __forceinline__ uint32_t orderedBits(float x) {
  const uint32_t b = floatBits(x);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__host__ __device__ __forceinline__ float orderedFloat(uint32_t o) {
  return bitsFloat((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

// ---------------------------------------------------------------------------
// Tiles.
//
// Points are processed in tiles of 128 consecutive points (in spatial order).
// The tile is the unit of the distance engine (a 128 x 128 block of pairs),
// of pruning (a bounding box per tile) and of the BVH leaves.
constexpr int kTile = 128;

inline int numTilesFor(int n) { return (n + kTile - 1) / kTile; }

// Entries of a per-position array padded to whole tiles: the passes copy a
// tile's 128 entries with one bulk copy, which must stay inside the
// allocation. Padding entries are never used as data.
inline size_t paddedToTiles(int n) { return (size_t)numTilesFor(n) * kTile; }

// Feature chunk width of the tiled point layout: features are stored per
// tile in chunks of KC (4/8/16/32), feature-major within a chunk, zero padded.
inline int chunkWidthFor(int d) { return d <= 4 ? 4 : d <= 8 ? 8 : d <= 16 ? 16 : 32; }
inline int numChunksFor(int d) {
  const int kc = chunkWidthFor(d);
  return (d + kc - 1) / kc;
}

// ---------------------------------------------------------------------------
// Device memory from the stream-ordered pool: after the first call of a
// given size, allocations are pool hits and cost microseconds.
template <typename T> struct DeviceBuffer {
  T *ptr = nullptr;
  size_t count = 0;
  cudaStream_t stream = 0;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  int allocate(size_t n, cudaStream_t s) {
    release();
    stream = s;
    count = n;
    if (n == 0)
      return 0;
    return (int)cudaMallocAsync((void **)&ptr, n * sizeof(T), s);
  }
  void release() {
    if (ptr)
      cudaFreeAsync(ptr, stream);
    ptr = nullptr;
    count = 0;
  }
  ~DeviceBuffer() { release(); }
  T *get() const { return ptr; }
  size_t bytes() const { return count * sizeof(T); }
};

// Iteration limit for every spin-wait in this library's kernels. A wait that
// runs out records kErrorTimeout in the kernel's error word and returns.
constexpr long long kSpinLimit = 1ll << 26;

} // namespace cuhc
