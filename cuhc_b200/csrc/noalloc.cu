// cuhc_pairwise_distances_noalloc: the pairwise-distance kernel for callers
// that cannot allocate GPU memory.
//
// Some callers can't call cudaMalloc: code that runs inside a host framework
// which owns every device allocation (a plugin given pre-sized buffers), code
// on a latency-critical path where an allocation could block or fail, and
// processes whose memory budget is fixed up front. This entry point takes the
// caller's device input and output buffers and allocates nothing itself: the
// scratch the kernel needs (the tiled copies of A and B that the distance
// engine reads) lives in one file-scope device array of fixed size,
// kNoAllocScratchBytes (32 MiB). Every GPU that loads the library holds that
// array until the process exits.
//
// Set-up: the first call on each device looks up the array's device address
// with cudaGetSymbolAddress (in host code the array's name is only a host-side
// stand-in, not a device address) and caches it per device; make that first
// call before any stream capture on the device.
//
// Sharing: every call uses the same array and it keeps the last call's
// contents, so the padding that must be zero is cleared on every call, and
// calls whose work overlaps on the GPU (different streams, or threads without
// ordering) race on the array. Order the calls, e.g. on one stream.
#include <mutex>

#include "metrics.cuh"
#include "pairwise.cuh"
#include "profiling.cuh"

namespace cuhc {
namespace {

constexpr size_t kNoAllocScratchBytes = 32u << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char gNoAllocScratch[kNoAllocScratchBytes];

std::mutex gScratchMutex;
void *gScratchAddress[kMaxDevices] = {};

// The device address of the scratch array on the current device.
int scratchAddress(void **out) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess)
    return (int)e;
  if (device < 0 || device >= kMaxDevices)
    return (int)cudaErrorInvalidDevice; // beyond the per-device address cache
  std::lock_guard<std::mutex> lock(gScratchMutex);
  if (!gScratchAddress[device]) {
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, gNoAllocScratch);
    if (e != cudaSuccess)
      return (int)e;
    gScratchAddress[device] = ptr;
  }
  *out = gScratchAddress[device];
  return 0;
}

// Row-major points -> the engine's tiled layout ([tile][d_pad][128]).
__global__ void tileRows(const float *__restrict__ points, int n, int d, int dPad,
                         float *__restrict__ tiled) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= (long long)n * d)
    return;
  const int p = (int)(e / d), f = (int)(e % d);
  tiled[((size_t)(p / kTile) * dPad + f) * kTile + p % kTile] = points[e];
}

} // namespace
} // namespace cuhc

extern "C" {

// Same result as cuhc_pairwise_distances (bit for bit), with device pointers
// and no allocation. A, B (B == NULL means B = A) and the nA x nB output are
// DEVICE memory of the current device (B == NULL needs nB == nA); stream
// may be NULL (default stream).
// The work is enqueued on `stream`; the call returns without waiting for it.
// Limit: the tiled copies of A and B must fit the 32 MiB scratch array,
// (ceil(nA/128) + ceil(nB/128)) * 128 * dPad * 4 bytes, dPad = d rounded up to
// the chunk width (4, 8, 16 or a multiple of 32); larger inputs return
// CUHC_ERROR_TOO_LARGE.
int cuhc_pairwise_distances_noalloc(const float *devA, int nA, const float *devB, int nB, int d,
                                    int metricId, float p, float *devOut, void *stream) {
  using namespace cuhc;
  if (nA <= 0 || nB <= 0 || d <= 0 || (!devB && nB != nA))
    return kErrorInvalidShape;
  if (metricId < kEuclidean || metricId > kCosine)
    return kErrorInvalidMetric;
  const int dPad = numChunksFor(d) * chunkWidthFor(d);
  const size_t floatsA = (size_t)numTilesFor(nA) * kTile * dPad;
  const size_t floatsB = devB ? (size_t)numTilesFor(nB) * kTile * dPad : 0;
  if ((floatsA + floatsB) * sizeof(float) > kNoAllocScratchBytes)
    return kErrorTooLarge;
  void *base = nullptr;
  const int status = scratchAddress(&base);
  if (status != 0)
    return status;
  cudaStream_t s = (cudaStream_t)stream;
  float *tiledA = (float *)base;
  float *tiledB = devB ? tiledA + floatsA : tiledA;
  // The array keeps the previous call's data: zero the padding lanes.
  cudaError_t e = cudaMemsetAsync(base, 0, (floatsA + floatsB) * sizeof(float), s);
  if (e != cudaSuccess)
    return (int)e;
  tileRows<<<(int)(((long long)nA * d + 255) / 256), 256, 0, s>>>(devA, nA, d, dPad, tiledA);
  noteLaunch();
  if (devB) {
    tileRows<<<(int)(((long long)nB * d + 255) / 256), 256, 0, s>>>(devB, nB, d, dPad, tiledB);
    noteLaunch();
  }
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return (int)e;
  return withMetric(metricId, p, [&](auto m) {
    return launchPairwise(tiledA, tiledB, nA, nB, d, m, devOut, s);
  });
}

} // extern "C"
