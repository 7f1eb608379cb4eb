#include "profiling.cuh"

#include <cmath>

#include "common.cuh"

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
__device__ unsigned long long gScreenAuditArray[kNumAuditWords];

namespace {
std::atomic<int> gAudit{0};
} // namespace

unsigned long long *screenAuditWords() {
  if (gAudit.load() == 0)
    return nullptr;
  void *ptr = nullptr;
  if (cudaGetSymbolAddress(&ptr, gScreenAuditArray) != cudaSuccess)
    return nullptr;
  return static_cast<unsigned long long *>(ptr);
}

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

// Screen audit on (1) or off (0); test and measurement hook, off by default
// (an audited pass evaluates every pair of its tiles twice more, in FP32 and
// FP64). Results of the passes never change.
int cuhc_set_screen_audit(int on) {
  if (on < 0 || on > 1)
    return cuhc::kErrorInvalidAlgorithm;
  cuhc::gAudit.store(on);
  return 0;
}

// The audit words of the current device since the last call, decoded (first
// `count` of): pairs, violations, min slack, max bound gap (relative to the
// norms), max bound gap (absolute), max exact abs error, max exact rel error;
// NaN where nothing was observed. Resets them.
int cuhc_screen_audit(double *out, int count) {
  unsigned long long host[cuhc::kNumAuditWords] = {};
  cudaError_t e = cudaMemcpyFromSymbol(host, cuhc::gScreenAuditArray, sizeof(host));
  if (e == cudaSuccess) {
    const unsigned long long zero[cuhc::kNumAuditWords] = {};
    e = cudaMemcpyToSymbol(cuhc::gScreenAuditArray, zero, sizeof(zero));
  }
  for (int i = 0; i < count && i < cuhc::kNumAuditWords; ++i) {
    const unsigned long long v = host[i];
    if (i == cuhc::kAuditPairs || i == cuhc::kAuditViolations)
      out[i] = (double)v;
    else if (v == 0)
      out[i] = NAN;
    else if (i == cuhc::kAuditMinSlack)
      out[i] = cuhc::orderedFloat(~(uint32_t)v);
    else
      out[i] = cuhc::orderedFloat((uint32_t)v);
  }
  return (int)e;
}

} // extern "C"
