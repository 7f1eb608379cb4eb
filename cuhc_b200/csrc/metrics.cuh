// Distance metrics and edge weights of the exact-clustering engine.
//
// A metric folds the features of a pair into an accumulator, one feature at
// a time in feature order 0..d-1, and finalizes it into the distance. The
// per-feature arithmetic of every metric is the reference's
// (distances.cuh:21-83), so every distance here is bit-identical to the
// reference's: the same FP32 operations in the same order. The engine only
// changes WHICH pairs are evaluated exactly, never how.
//
// Two additions serve the hot loop:
//   filter(acc)        a cheap monotone proxy of the distance, read straight
//                      from the accumulator (no sqrt, no division);
//   filterBound(dist)  a conservative bound: finalize(acc) <= dist implies
//                      filter(acc) <= filterBound(dist).
// A pair whose filter value exceeds the bound of the row's current best can
// not win, so the exact epilogue (sqrt, weight, key compare) runs only for
// the few pairs that pass. Metrics with a tensor-core screen (screen.cuh)
// also give
//   screenBound(dist)  the bound on the screened value: the screen's value of
//                      a pair is at most its exact value's image here, so a
//                      pair with distance <= dist has screened value <=
//                      screenBound(dist) (the squared distance for the
//                      Euclidean metrics, the distance itself for cosine).
//
// Every built-in metric treats a zero-padded feature pair (0, 0) as an exact
// no-op (fmaf(0,0,acc) == acc, acc + |0| == acc, fmax(acc, 0) == acc for
// acc >= 0, the Minkowski guard x > 0), which the tiled layout relies on.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "common.cuh"

namespace cuhc {

#define CUHC_HD __host__ __device__ __forceinline__

// Largest float whose sqrtf can still be <= dist, rounded up: if
// sqrtf(s) <= dist then s <= sqBound(dist).
__device__ __forceinline__ float sqBound(float dist) {
  if (!(dist < INFINITY))
    return INFINITY;
  const float up = nextafterf(dist, INFINITY);
  return __fmul_ru(up, up);
}

struct SqEuclideanMetric {
  using Acc = float;
  static constexpr bool kBoxBound = true;
  static constexpr bool kHasFilter = true;
  // Two columns per instruction (Blackwell's packed FP32): each lane is the
  // same IEEE subtraction and fused multiply-add as accumulate(), and
  // (b - a)^2 == (a - b)^2 exactly, so the bits are those of the scalar fold.
  static constexpr bool kPacked = true;
  CUHC_HD Acc init() const { return 0.0f; }
  CUHC_HD Acc accumulate(Acc acc, float a, float b) const {
    const float diff = a - b;
    return fmaf(diff, diff, acc);
  }
  __device__ __forceinline__ float2 accumulate2(float2 acc, float2 negA, float2 b) const {
    const float2 diff = __fadd2_rn(b, negA);
    return __ffma2_rn(diff, diff, acc);
  }
  CUHC_HD Acc combine(Acc x, Acc y) const { return x + y; }
  CUHC_HD float finalize(Acc acc) const { return acc; }
  __device__ __forceinline__ float filter(Acc acc) const { return acc; }
  __device__ __forceinline__ float filterBound(float dist) const { return dist; }
  __device__ __forceinline__ float screenBound(float dist) const { return dist; }
};

struct EuclideanMetric : SqEuclideanMetric {
  CUHC_HD float finalize(Acc acc) const { return sqrtf(acc); }
  __device__ __forceinline__ float filterBound(float dist) const { return sqBound(dist); }
  __device__ __forceinline__ float screenBound(float dist) const { return sqBound(dist); }
};

struct ManhattanMetric {
  using Acc = float;
  static constexpr bool kBoxBound = true;
  static constexpr bool kHasFilter = true;
  static constexpr bool kPacked = false;
  CUHC_HD Acc init() const { return 0.0f; }
  CUHC_HD Acc accumulate(Acc acc, float a, float b) const { return acc + fabsf(a - b); }
  CUHC_HD Acc combine(Acc x, Acc y) const { return x + y; }
  CUHC_HD float finalize(Acc acc) const { return acc; }
  __device__ __forceinline__ float filter(Acc acc) const { return acc; }
  __device__ __forceinline__ float filterBound(float dist) const { return dist; }
};

struct ChebyshevMetric {
  using Acc = float;
  static constexpr bool kBoxBound = true;
  static constexpr bool kHasFilter = true;
  static constexpr bool kPacked = false;
  CUHC_HD Acc init() const { return 0.0f; }
  CUHC_HD Acc accumulate(Acc acc, float a, float b) const { return fmaxf(acc, fabsf(a - b)); }
  CUHC_HD Acc combine(Acc x, Acc y) const { return fmaxf(x, y); }
  CUHC_HD float finalize(Acc acc) const { return acc; }
  __device__ __forceinline__ float filter(Acc acc) const { return acc; }
  __device__ __forceinline__ float filterBound(float dist) const { return dist; }
};

// |x|^p per feature through exp2/log2, as the reference's device code does
// (distances.cuh:50-66): the same operations give the same bits.
struct MinkowskiMetric {
  float p;
  using Acc = float;
  static constexpr bool kBoxBound = true;
  static constexpr bool kHasFilter = true;
  static constexpr bool kPacked = false;
  CUHC_HD Acc init() const { return 0.0f; }
  CUHC_HD Acc accumulate(Acc acc, float a, float b) const {
    const float x = fabsf(a - b);
#ifdef __CUDA_ARCH__
    return x > 0.0f ? acc + exp2f(p * __log2f(x)) : acc;
#else
    return acc + powf(x, p);
#endif
  }
  CUHC_HD Acc combine(Acc x, Acc y) const { return x + y; }
  CUHC_HD float finalize(Acc acc) const { return powf(acc, 1.0f / p); }
  __device__ __forceinline__ float filter(Acc acc) const { return acc; }
  // powf's error is a few ulp; 1e-3 relative is far beyond it.
  __device__ __forceinline__ float filterBound(float dist) const {
    return dist < INFINITY ? powf(dist, p) * 1.001f + 1e-30f : INFINITY;
  }
};

struct CosineMetric {
  using Acc = float3;
  static constexpr bool kBoxBound = false;
  static constexpr bool kHasFilter = false;
  static constexpr bool kPacked = false;
  CUHC_HD Acc init() const { return make_float3(0.0f, 0.0f, 0.0f); }
  CUHC_HD Acc accumulate(Acc acc, float a, float b) const {
    acc.x = fmaf(a, b, acc.x);
    acc.y = fmaf(a, a, acc.y);
    acc.z = fmaf(b, b, acc.z);
    return acc;
  }
  CUHC_HD Acc combine(Acc x, Acc y) const {
    return make_float3(x.x + y.x, x.y + y.y, x.z + y.z);
  }
  CUHC_HD float finalize(Acc acc) const {
    const float denom = sqrtf(acc.y * acc.z);
    return denom > 0.0f ? 1.0f - acc.x / denom : 1.0f;
  }
  // No cheap monotone proxy: every pair takes the exact path.
  __device__ __forceinline__ float filter(Acc) const { return 0.0f; }
  __device__ __forceinline__ float filterBound(float) const { return INFINITY; }
  // The screen bounds the distance itself.
  __device__ __forceinline__ float screenBound(float dist) const { return dist; }
};

// Relative slack of the box lower bound: a pair's computed distance and the
// computed bound can each be off by about d rounding steps (more for the
// fast Minkowski powers); this margin is far above that and far too small to
// cost pruning. Same margin as the reference (spatial.cuh:183-185).
CUHC_HD float boxSlack(int d) { return 1e-5f + (d + 8) * 5e-7f; }

// ---------------------------------------------------------------------------
// Edge weights: what an (i, j) pair weighs given its distance and a
// per-point value (nothing, the core distance, the cluster size).
//
//   weight(d, vi, vj)            exact weight, the reference's formula;
//   distBound(thr, vi)           conservative: weight(d, vi, vj) <= thr for
//                                some vj implies d <= distBound(thr, vi);
//   lowerBound(dlb, vI, vJ)      weight lower bound of a tile pair from a
//                                distance lower bound and the tiles' smallest
//                                values (used with the slack);
//   feasible(thr, vi)            false if no pair of row i can weigh <= thr.

struct PlainWeight {
  const float *value = nullptr; // unused
  __device__ __forceinline__ float load(int) const { return 0.0f; }
  __device__ __forceinline__ float weight(float d, float, float) const { return d; }
  __device__ __forceinline__ float distBound(float thr, float) const { return thr; }
  __device__ __forceinline__ float lowerBound(float dlb, float, float) const { return dlb; }
  __device__ __forceinline__ bool feasible(float, float) const { return true; }
};

// HDBSCAN's mutual reachability: max(core_i, core_j, d / alpha), with the
// reference's operation order (hdbscan.cuh:342-351).
struct MutualReachWeight {
  const float *value = nullptr; // core distances, by position
  float alpha = 1.0f;
  __device__ __forceinline__ float load(int i) const { return value[i]; }
  __device__ __forceinline__ float weight(float d, float ci, float cj) const {
    return fmaxf(fmaxf(ci, cj), alpha == 1.0f ? d : d / alpha);
  }
  __device__ __forceinline__ float distBound(float thr, float) const {
    if (!(thr < INFINITY))
      return INFINITY;
    return alpha == 1.0f ? thr : __fmul_ru(__fmul_ru(thr, alpha), 1.0000005f);
  }
  __device__ __forceinline__ float lowerBound(float dlb, float cI, float cJ) const {
    return fmaxf(fmaxf(cI, cJ), alpha == 1.0f ? dlb : dlb / alpha);
  }
  __device__ __forceinline__ bool feasible(float thr, float ci) const { return ci <= thr; }
};

// Ward's selection weight on squared distances between centroids, with the
// reference's fast division (rnn_ward.cuh:56-64): the same intrinsic on the
// same operands gives the same bits, and it is symmetric in (i, j).
struct WardWeight {
  const float *value = nullptr; // cluster sizes as floats, by slot
  __device__ __forceinline__ float load(int i) const { return value[i]; }
  __device__ __forceinline__ float weight(float s, float si, float sj) const {
    return __fdividef(2.0f * (si * sj) * s, si + sj);
  }
  // 2 si sj s / (si + sj) <= thr  =>  s <= thr (1/si + 1/sj) / 2, and
  // sj >= 1. The fast division is within 2 ulp; 1e-5 covers it.
  __device__ __forceinline__ float distBound(float thr, float si) const {
    if (!(thr < INFINITY))
      return INFINITY;
    return __fmul_ru(thr, (1.0f / si + 1.0f) * 0.5f * 1.00001f);
  }
  __device__ __forceinline__ float lowerBound(float slb, float sI, float sJ) const {
    return 2.0f * sI * sJ / (sI + sJ) * slb * 0.9999f;
  }
  __device__ __forceinline__ bool feasible(float, float) const { return true; }
};

// Metric ids of the C ABI; the reference's table (capi.cu:17-24).
enum MetricId : int {
  kEuclidean = 0,
  kSqEuclidean = 1,
  kManhattan = 2,
  kChebyshev = 3,
  kMinkowski = 4,
  kCosine = 5,
};

// Calls run(metric) with the metric object for metricId.
template <typename Run> int withMetric(int metricId, float p, Run run) {
  switch (metricId) {
  case kEuclidean:
    return run(EuclideanMetric{});
  case kSqEuclidean:
    return run(SqEuclideanMetric{});
  case kManhattan:
    return run(ManhattanMetric{});
  case kChebyshev:
    return run(ChebyshevMetric{});
  case kMinkowski:
    return run(MinkowskiMetric{p});
  case kCosine:
    return run(CosineMetric{});
  default:
    return kErrorInvalidMetric;
  }
}

} // namespace cuhc
