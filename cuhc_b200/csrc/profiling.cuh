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

// Screen audit (cuhc_set_screen_audit): with it on, every screened tile also
// checks each valid pair's tensor-core value D' against the reference FP32
// squared distance s and an FP64 recomputation s64, and folds the results
// into these device words: pairs audited, pairs with D' > s + 2^-70 (the
// screen's guarantee broken; must stay 0), then minima / maxima stored as
// order-preserving float bits (min: complemented) of
//   slack      (s - D') / (e (|x|^2 + |y|^2)), x, y the centred coordinates
//              and e the screen's margin, over the pairs whose margin
//              e (|x|^2 + |y|^2) exceeds the absolute 2^-70; >= 0 is the
//              guarantee, and the margin is twice the modelled error, so
//              about 0.5 or more means the error model holds with room;
//   boundGap   (s64 - D') / (|x|^2 + |y|^2): how far below the exact value
//              the screened bound sits, relative to the norms;
//   boundAbs   s64 - D';
//   exactAbs   |s - s64| and exactRel |s - s64| / s64 (s64 > 0): the
//              reference FP32 chain's own error.
enum ScreenAuditWord : int { kAuditPairs = 0, kAuditViolations = 1, kAuditMinSlack = 2,
                             kAuditMaxBoundGap = 3, kAuditMaxBoundAbs = 4, kAuditMaxExactAbs = 5,
                             kAuditMaxExactRel = 6, kNumAuditWords = 7 };
// Null when the audit is off.
unsigned long long *screenAuditWords();

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
