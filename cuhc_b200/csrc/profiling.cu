#include "profiling.cuh"

#include <atomic>
#include <mutex>

namespace cuhc {
namespace {
std::atomic<unsigned long long> gLaunches{0};
std::atomic<int> gTiming{0};
std::mutex gTimerMutex;
double gMs[kNumTimers] = {};
unsigned long long gCount[kNumTimers] = {}, gTiles[kNumTimers] = {};
} // namespace

__device__ unsigned long long gScreenCounterArray[kNumScreenCounters];

void noteLaunch(int count) { gLaunches.fetch_add((unsigned long long)count); }
bool timingEnabled() { return gTiming.load() != 0; }

unsigned long long *screenCounters() {
  if (!timingEnabled())
    return nullptr;
  void *ptr = nullptr;
  if (cudaGetSymbolAddress(&ptr, gScreenCounterArray) != cudaSuccess)
    return nullptr;
  return static_cast<unsigned long long *>(ptr);
}

PassTimer::PassTimer(int k, cudaStream_t s) : kind(k), stream(s) {
  if (k < 0 || !timingEnabled())
    return; // kind -1: a launch that is not timed (e.g. inside a stream capture)
  cudaEventCreate(&start);
  cudaEventCreate(&stop);
  cudaEventRecord(start, stream);
}

void PassTimer::finish(unsigned long long tilesComputed) {
  if (!start)
    return;
  cudaEventRecord(stop, stream);
  cudaEventSynchronize(stop);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, start, stop);
  std::lock_guard<std::mutex> lock(gTimerMutex);
  gMs[kind] += ms;
  gCount[kind] += 1;
  gTiles[kind] += tilesComputed;
}

PassTimer::~PassTimer() {
  if (start)
    cudaEventDestroy(start);
  if (stop)
    cudaEventDestroy(stop);
}

} // namespace cuhc

extern "C" {

unsigned long long cuhc_launch_count(void) { return cuhc::gLaunches.load(); }

int cuhc_set_timing(int on) {
  cuhc::gTiming.store(on ? 1 : 0);
  return 0;
}

// Per pass kind (0 k-NN pass, 1 nearest pass, 2 screened nearest pass,
// 3 screened k-NN pass): summed
// device milliseconds, launches and tiles computed since the last call;
// resets them.
int cuhc_kernel_timing(double *ms, unsigned long long *launches, unsigned long long *tiles,
                       int count) {
  std::lock_guard<std::mutex> lock(cuhc::gTimerMutex);
  for (int i = 0; i < count && i < cuhc::kNumTimers; ++i) {
    ms[i] = cuhc::gMs[i];
    launches[i] = cuhc::gCount[i];
    tiles[i] = cuhc::gTiles[i];
    cuhc::gMs[i] = 0.0;
    cuhc::gCount[i] = cuhc::gTiles[i] = 0;
  }
  return 0;
}

// Screened-pass counters of the current device since the last call (first
// `count` of: exact rechecks, exact-path row visits, indicator tiles, masked
// tiles, tiles no row needed); resets them. Counted only while timing is on.
int cuhc_screen_counters(unsigned long long *out, int count) {
  unsigned long long host[cuhc::kNumScreenCounters] = {};
  cudaError_t e = cudaMemcpyFromSymbol(host, cuhc::gScreenCounterArray, sizeof(host));
  if (e == cudaSuccess) {
    const unsigned long long zero[cuhc::kNumScreenCounters] = {};
    e = cudaMemcpyToSymbol(cuhc::gScreenCounterArray, zero, sizeof(zero));
  }
  for (int i = 0; i < count && i < cuhc::kNumScreenCounters; ++i)
    out[i] = host[i];
  return (int)e;
}

} // extern "C"
