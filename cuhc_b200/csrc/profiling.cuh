// Optional per-kernel timing and launch counting.
//
// Kernel launches of this library go through noteLaunch(), so a caller can
// read how many of its kernels ran (cuhc_launch_count). With timing switched
// on (cuhc_set_timing), the all-pairs passes are bracketed by CUDA events on
// the stream they are launched on; their device time and the tiles they
// computed are summed per pass kind (cuhc_kernel_timing). Off by default:
// the events cost a few microseconds per pass.
#pragma once

#include <cuda_runtime.h>

namespace cuhc {

enum TimerKind : int { kTimerKnnPass = 0, kTimerNearestPass = 1, kTimerScreenPass = 2,
                       kTimerScreenKnnPass = 3, kNumTimers = 4 };

void noteLaunch(int count = 1);
bool timingEnabled();

// Screened-pass counters (device memory of the current device), summed by
// the screened kernels while timing is on: exact rechecks, row visits that
// took the exact path, tiles whose components were excluded by indicator
// slots, tiles masked by component in the epilogue, candidate tiles that no
// row of the block needed (skipped before any copy).
enum ScreenCounter : int { kScreenRechecks = 0, kScreenSlowRows = 1, kScreenIndicatorTiles = 2,
                           kScreenMaskedTiles = 3, kScreenPrefiltered = 4,
                           kNumScreenCounters = 5 };
// Null when timing is off (the kernels then count nothing).
unsigned long long *screenCounters();

// RAII bracket around one pass launch; records only when timing is on.
struct PassTimer {
  int kind;
  cudaStream_t stream;
  cudaEvent_t start = nullptr, stop = nullptr;
  PassTimer(int kind, cudaStream_t stream);
  // Call after the launch; accumulates device time (synchronizes the stop
  // event only when timing is on) and the pass's tile count.
  void finish(unsigned long long tilesComputed);
  ~PassTimer();
};

} // namespace cuhc
