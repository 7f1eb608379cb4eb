// The tensor-core screened pass: the nearest / k-NN passes of passes.cuh
// with the all-pairs distance work moved to tcgen05 MMAs.
//
// Screen. Per row tile the block centres every coordinate on the row tile's
// box centre c (x = a - c, y = b - c, FP32) and builds K-major TF32 operands
// such that one MMA accumulation gives, in tensor memory,
//     D'(i, j) = N_i + N_j - 2 sum_k tf32(x_k) tf32(y_k)   (+ 2^90, below)
// with N = (1 - e) |x|^2 split into two TF32 terms. The margin e
// (screenMargin) is twice a rigorous bound, as a multiple of |x|^2 + |y|^2,
// of every error involved: the one-term TF32 product (2^-10), the norms' FP32
// rounding and split, the centring rounding, the tensor core's FP32
// accumulation (modelled as 2^-22 of the sum of absolute products per
// addition, four times over) and the reference's own FP32 rounding of the
// squared distance s. Hence D'(i, j) <= s(i, j) for every pair of different
// components, and a pair can only pass its row's filter bound F (a bound on
// s) if D'(i, j) <= F + 2^-70 (the absolute term covers subnormal products
// that the tensor core may flush). Exactly those pairs are recomputed with
// the reference's FP32 chain from the raw coordinates, so every weight, key
// and k-th distance is bit-identical to the plain pass. The screen needs
// every coordinate extent <= 2^40 (nothing overflows); wider data runs plain.
//
// Component indicators. In Borůvka rounds a row's own component must not
// count. When the row tile holds at most R distinct components (R = the K
// slots left after coordinates and norms, >= 4), slot q of row i holds 2^90
// if comp(i) is the q-th of them and slot q of column j holds 1 if comp(j)
// is: the MMA adds 2^90 to every same-component pair and exactly 0 to every
// other pair, and the epilogue takes a plain row minimum. Otherwise the
// epilogue masks by component.
//
// Pipeline, warp-specialised, one row tile per block:
//   producer warp 6: picks the next candidate tile (32 list entries per
//     step) and lane 0 issues its bulk copies (raw coordinates + metadata)
//     into a ring of `stages` slots, at most `lead` ordinals beyond the last
//     one every consumer warp has finished;
//   MMA warp 7 (one thread): issues the MMA of each tile as soon as its
//     accumulator and its column operand are ready;
//   builder warps 4-5: build the column operand of each staged tile (two
//     columns per thread) as soon as the MMA that last read its buffer is
//     done;
//   consumer warps 0-3 (row i = thread = tensor-memory lane): read the
//     accumulator (row minimum, and candidate bits when some row may gain),
//     release it, recheck rows with a pair at or below their filter, release
//     the ring slot, refresh the row threshold when it may have changed.
// Tensor memory holds two 128 x 128 FP32 accumulators, so the MMAs of tile
// t + 1 run while the consumers read tile t; since a warp releases the
// accumulator before its exact path, one warp's rechecks delay the others
// only once it falls behind by the ring's slack. mbarriers link the stages:
// rawFull (copy landed), opBReady (operand built), mmaFull (MMA done + slot
// info), tmemEmpty (every consumer warp has read the accumulator), rawEmpty
// (every consumer warp done with the ring slot). Candidate collection and ordering
// are those of passes.cuh, one batch at a time; a sentinel ordinal ends each
// batch. Every wait is bounded; one that runs out marks the block failed,
// every later wait gives up at once, and the pass returns kErrorTimeout.
#pragma once

#include <algorithm>
#include <climits>
#include <cmath>
#include <type_traits>

#include "passes.cuh"
#include "umma.cuh"

namespace cuhc {

// K of the screened product for chunk width KC: KC coordinates, 4 norm
// terms and at least 4 component slots, a multiple of the MMA's K step (8).
__host__ __device__ constexpr int screenKPad(int kc) { return (kc + 8 + 7) / 8 * 8; }
__host__ __device__ constexpr int screenSlots(int kc) { return screenKPad(kc) - kc - 4; }
// Ring of staged column tiles: `stages` slots (chosen per launch, as many as
// keep two blocks on an SM, kScreenMinStages .. kScreenMaxStages). The
// producer issues ordinal o once every consumer warp has finished ordinal
// o - lead, lead = min(stages - 1, screenLead(KC)): copies run that far ahead
// of the slowest consumer warp, and a tile is picked against thresholds at
// most that many tiles old.
__host__ __device__ constexpr int screenLead(int kc) { return kc <= 8 ? 5 : 4; }
constexpr int kScreenMinStages = 5;
constexpr int kScreenMaxStages = 8;
constexpr int kScreenMaxSlots = 8;
constexpr int kBuilderWarps = 2; // warps 4..5 build column operands
constexpr int kBuilderThreads = 32 * kBuilderWarps;
constexpr int kProducerWarp = 6; // picks candidate tiles and issues their bulk copies
constexpr int kMmaWarp = 7;      // issues the MMAs
constexpr int kFirstPhase = 64;  // tiles of a batch's first phase (then x8 per phase)
constexpr float kIndicator = 0x1p90f;
constexpr float kScreenAbsSlack = 0x1p-70f;
constexpr float kScreenMaxExtent = 0x1p40f;

// Cosine. The screen runs on unit vectors: x^ = a rsqrt(|a|^2) (0 for a zero
// point), y^ likewise, and one MMA gives D'(i, j) = c - sum_k tf32(x^_k)
// tf32(y^_k) with c = 1 - e rounded down to TF32. e (screenMarginCosine) is
// twice a bound of every error against the reference's FP32 distance
// 1 - (a.b) / sqrt(|a|^2 |b|^2) (distances.cuh:69-83): the TF32 products, the
// normalisation, the tensor core's accumulation (modelled as for the
// Euclidean screen) and the reference's own rounding (dot product, norms,
// square root, division, 1 - q), all relative to sum |x^_k y^_k| + 1 <= 2
// (Cauchy-Schwarz). Hence D' <= the reference's distance for every pair,
// provided no norm product underflows or overflows there (the reference then
// returns 1 whatever the angle): the screen needs every nonzero point's
// squared norm in [2^-60, 2^60] (SpatialIndex::normsWithin); other data runs
// plain. A zero point screens at c < 1, its reference distance being 1.
constexpr float kCosineNormLow = 0x1p-60f;
constexpr float kCosineNormHigh = 0x1p60f;

inline float screenMarginCosine(int d, int kc) {
  const double u = std::ldexp(1.0, -24), t = std::ldexp(1.0, -11), u22 = std::ldexp(1.0, -22);
  const double product = t * (2.0 + t);                 // tf32(x^) tf32(y^) against x^ y^
  const double normalise = 8.0 * u;                     // rsqrtf (2 ulp) and the scaling
  const double mma = 4.0 * screenKPad(kc) * u22 * 2.01; // accumulation, four times over
  const double reference = (2.0 * d + 8.0) * u;         // the reference's FP32 chain
  return (float)(2.0 * (product + normalise + mma + reference));
}

// e of the header comment, for d features staged as chunks of kc.
inline float screenMargin(int d, int kc) {
  const double u = std::ldexp(1.0, -24), t = std::ldexp(1.0, -11), u22 = std::ldexp(1.0, -22);
  const double product = t * (2.0 + t);                 // tf32(x) tf32(y) against x y
  const double norms = 1.01 * kc * u + u + u22;         // |x|^2 in FP32, times (1 - e), split
  const double mma = 4.0 * screenKPad(kc) * u22 * 2.01; // accumulation, four times over
  const double centring = 4.0 * u;                      // a - c and b - c rounded
  const double reference = 2.02 * (d + 3) * u;          // the reference's FP32 chain
  return (float)(2.0 * (product + norms + mma + centring + reference));
}

// A k-NN list entry of the screened pass: value bits << 32 | position, so
// that one 64-bit move carries both and keys order by value (values are
// clamped at +0, so their bits order like the floats), then by position. An
// empty entry holds +inf.
constexpr unsigned long long kEmptyListKey = 0x7f800000ffffffffull;

__device__ __forceinline__ float listKeyValue(unsigned long long key) {
  return __uint_as_float((uint32_t)(key >> 32));
}

// Inserts `key` (its value below the k-th, whose entry leaves the list) into
// a row's ascending key list, after every entry <= key; walks down from the
// end four entries at a time, as insertSortedPos does.
__device__ __forceinline__ void insertListKey(unsigned long long *list, int k,
                                              unsigned long long key) {
  int i = k - 1;
  for (; i >= 4; i -= 4) {
    const unsigned long long a = list[i - 1], b = list[i - 2], c = list[i - 3], d = list[i - 4];
    if (!(a > key))
      goto place;
    list[i] = a;
    if (!(b > key)) {
      i -= 1;
      goto place;
    }
    list[i - 1] = b;
    if (!(c > key)) {
      i -= 2;
      goto place;
    }
    list[i - 2] = c;
    if (!(d > key)) {
      i -= 3;
      goto place;
    }
    list[i - 3] = d;
  }
  for (; i > 0 && list[i - 1] > key; --i)
    list[i] = list[i - 1];
place:
  list[i] = key;
}

// k-NN, the row tile against itself (every list still empty): a bound on the
// screened value of every pair that can enter the row's list, so that only
// those pairs are rechecked instead of all 128. With T the k-th smallest
// screened value D' over the tile's valid columns (bisected to within 2^-8 of
// the value range, from above), the k columns of smallest D' all have exact
// values s <= D' + delta <= T + delta (delta bounds s - D' for every pair of the
// tile), so the row's k-th smallest exact value in the tile, and every pair
// that can still enter its list, has D' <= s <= T + delta. +inf when the tile
// holds fewer than k valid columns. Whole warp (tensor-memory loads).
__device__ __forceinline__ float selfTileBound(uint32_t taddr, const int *cOrig, int firstCol,
                                               int n, int k, float delta) {
  const int lane = threadIdx.x & 31;
  uint32_t valid[4];
  int count = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    valid[q] = __ballot_sync(0xffffffffu,
                             firstCol + q * 32 + lane < n && cOrig[q * 32 + lane] >= 0);
    count += __popc(valid[q]);
  }
  if (count < k)
    return INFINITY;
  float lo = INFINITY, hi = -INFINITY;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float v[32];
    tmemLoad32(taddr + q * 32, v);
#pragma unroll
    for (int c = 0; c < 32; ++c)
      if ((valid[q] >> c) & 1u) {
        lo = fminf(lo, v[c]);
        hi = fmaxf(hi, v[c]);
      }
  }
  // Invariant: at least k valid values are <= hi.
#pragma unroll 1
  for (int step = 0; step < 8; ++step) {
    const float mid = 0.5f * (lo + hi);
    int below = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      float v[32];
      tmemLoad32(taddr + q * 32, v);
#pragma unroll
      for (int c = 0; c < 32; ++c)
        below += (((valid[q] >> c) & 1u) && v[c] <= mid) ? 1 : 0;
    }
    if (below >= k)
      hi = mid;
    else
      lo = mid;
  }
  return hi + delta;
}

// Dynamic shared memory of a screened block with `stages` ring slots, in
// floats from the base (every region 16-byte aligned).
template <int KC> struct ScreenLayout {
  static constexpr int kPad = screenKPad(KC);
  static constexpr size_t rawFloats = (size_t)KC * kTile;
  static constexpr size_t metaInts = 3 * kTile; // orig, comp, value
  int stages;
  __host__ __device__ size_t sA() const { return 0; }
  __host__ __device__ size_t raw() const { return rawFloats; }
  __host__ __device__ size_t meta() const { return raw() + stages * rawFloats; }
  __host__ __device__ size_t opA() const { return meta() + stages * metaInts; }
  __host__ __device__ size_t opB() const { return opA() + (size_t)kTile * kPad; }
  // Row box low, high, centre (KC each).
  __host__ __device__ size_t box() const { return opB() + 2 * (size_t)kTile * kPad; }
  // k-NN lists: k 64-bit keys per row (value bits << 32 | position); 8-byte
  // aligned since KC is even.
  __host__ __device__ size_t lists() const { return box() + 3 * KC; }
  __host__ __device__ size_t bytes(int k) const {
    return (lists() + (size_t)kTile * k * 2) * sizeof(float);
  }
};

struct ScreenSync {
  uint64_t rawFull[kScreenMaxStages], rawEmpty[kScreenMaxStages];
  uint64_t mmaFull[2], tmemEmpty[2], opBReady[2];
  int rawTile[kScreenMaxStages]; // column tile (| kPureColumnTile) per ring slot, -1 ends the batch
  int slotTile[2];            // the same, per accumulator
  float warpThr[4];
  float rowF[kTile]; // each row's filter bound as last refreshed (-inf: gains nothing)
  float groupF[4];   // the largest rowF of each consumer warp's 32 rows
  int cursor, batchDone; // the producer's place in the candidate list at a phase end
  int rowSet[kScreenMaxSlots];
  int rowSetCount, oneHot, failed;
  uint32_t tmemBase;
};

__device__ __forceinline__ float min3(float a, float b, float c) {
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// Bounded wait that gives up at once when the block already failed; false
// when it did not see the phase complete.
__device__ __forceinline__ bool screenWait(uint64_t *bar, uint32_t parity, ScreenSync &ss) {
  if (*(volatile int *)&ss.failed)
    return false;
  if (mbarrierWait(bar, parity))
    return true;
  *(volatile int *)&ss.failed = 1;
  return false;
}

// Stores the kPad operand values of one point (row of the K-major canonical
// layout: 8-row core matrices of 16-byte rows, LBO 128, SBO kPad * 32).
template <int kPad>
__device__ __forceinline__ void storeOperandRow(float *op, int row, const float (&val)[kPad]) {
  char *base = reinterpret_cast<char *>(op) + (size_t)(row >> 3) * (kPad * 32) + (row & 7) * 16;
#pragma unroll
  for (int q = 0; q < kPad / 4; ++q)
    *reinterpret_cast<float4 *>(base + q * 128) =
        make_float4(val[4 * q], val[4 * q + 1], val[4 * q + 2], val[4 * q + 3]);
}

// Row operand of row tile point i: [-2 x (KC), N hi, N lo, 1, 1, indicators]
// (the factor -2, exact, sits on the side built once per row tile).
template <int KC>
__device__ __forceinline__ void buildRowOperand(const float *sA, const float *centre, float scale,
                                                int i, bool valid, int comp,
                                                const ScreenSync &ss, float *opA) {
  constexpr int kPad = screenKPad(KC), R = screenSlots(KC);
  float val[kPad];
  float n = 0.0f;
#pragma unroll
  for (int k = 0; k < KC; ++k) {
    const float x = sA[k * kTile + i] - centre[k];
    n = fmaf(x, x, n);
    val[k] = -2.0f * toTf32(x);
  }
  const float ns = n * scale, nh = toTf32(ns);
  val[KC] = nh;
  val[KC + 1] = toTf32(ns - nh);
  val[KC + 2] = 1.0f;
  val[KC + 3] = 1.0f;
#pragma unroll
  for (int q = 0; q < R; ++q)
    val[KC + 4 + q] =
        (ss.oneHot && valid && q < ss.rowSetCount && comp == ss.rowSet[q]) ? kIndicator : 0.0f;
  storeOperandRow<kPad>(opA, i, val);
}

// Column operand of staged point j: [y (KC), 1, 1, N hi, N lo, indicators];
// the tile centre comes in registers.
template <int KC>
__device__ __forceinline__ void buildColumnOperand(const float *raw, const int *comp,
                                                   const float (&centre)[KC], float scale, int j,
                                                   bool oneHot, const ScreenSync &ss,
                                                   float *opB) {
  constexpr int kPad = screenKPad(KC), R = screenSlots(KC);
  float val[kPad];
  float n = 0.0f;
#pragma unroll
  for (int k = 0; k < KC; ++k) {
    const float y = raw[k * kTile + j] - centre[k];
    n = fmaf(y, y, n);
    val[k] = toTf32(y);
  }
  const float ns = n * scale, nh = toTf32(ns);
  val[KC] = 1.0f;
  val[KC + 1] = 1.0f;
  val[KC + 2] = nh;
  val[KC + 3] = toTf32(ns - nh);
  const int c = oneHot ? comp[j] : INT_MIN;
#pragma unroll
  for (int q = 0; q < R; ++q)
    val[KC + 4 + q] = (oneHot && q < ss.rowSetCount && c == ss.rowSet[q]) ? 1.0f : 0.0f;
  storeOperandRow<kPad>(opB, j, val);
}

// Cosine operands: the reciprocal norm of a point (0 for a zero point), its
// squared norm folded in feature order as the reference does.
template <int KC>
__device__ __forceinline__ float unitScale(const float *x, int stride, int i) {
  float n = 0.0f;
#pragma unroll
  for (int k = 0; k < KC; ++k)
    n = fmaf(x[k * stride + i], x[k * stride + i], n);
  return n > 0.0f ? rsqrtf(n) : 0.0f;
}

// Row operand of row tile point i (cosine): [-x^ (KC), 1, 0, 0, 0, indicators].
template <int KC>
__device__ __forceinline__ void buildRowOperandCosine(const float *sA, int i, bool valid, int comp,
                                                      const ScreenSync &ss, float *opA) {
  constexpr int kPad = screenKPad(KC), R = screenSlots(KC);
  float val[kPad];
  const float r = unitScale<KC>(sA, kTile, i);
#pragma unroll
  for (int k = 0; k < KC; ++k)
    val[k] = -toTf32(sA[k * kTile + i] * r);
  val[KC] = 1.0f;
  val[KC + 1] = 0.0f;
  val[KC + 2] = 0.0f;
  val[KC + 3] = 0.0f;
#pragma unroll
  for (int q = 0; q < R; ++q)
    val[KC + 4 + q] =
        (ss.oneHot && valid && q < ss.rowSetCount && comp == ss.rowSet[q]) ? kIndicator : 0.0f;
  storeOperandRow<kPad>(opA, i, val);
}

// Column operand of staged point j (cosine): [y^ (KC), c, 0, 0, 0,
// indicators], c = 1 - e rounded down to TF32.
template <int KC>
__device__ __forceinline__ void buildColumnOperandCosine(const float *raw, const int *comp,
                                                         float c, int j, bool oneHot,
                                                         const ScreenSync &ss, float *opB) {
  constexpr int kPad = screenKPad(KC), R = screenSlots(KC);
  float val[kPad];
  const float r = unitScale<KC>(raw, kTile, j);
#pragma unroll
  for (int k = 0; k < KC; ++k)
    val[k] = toTf32(raw[k * kTile + j] * r);
  val[KC] = c;
  val[KC + 1] = 0.0f;
  val[KC + 2] = 0.0f;
  val[KC + 3] = 0.0f;
  const int cj = oneHot ? comp[j] : INT_MIN;
#pragma unroll
  for (int q = 0; q < R; ++q)
    val[KC + 4 + q] = (oneHot && q < ss.rowSetCount && cj == ss.rowSet[q]) ? 1.0f : 0.0f;
  storeOperandRow<kPad>(opB, j, val);
}

// Audit of one computed tile (cuhc_set_screen_audit; one consumer warp, its
// accumulator still held): every valid pair of the warp's rows -- a real
// column point, and in Borůvka passes another component -- has its screened
// value D' compared with the reference FP32 squared distance s (the chain the
// exact path recomputes) and with an FP64 recomputation s64; the warp folds
// the pair count, violations (D' > s + 2^-70) and the extrema described at
// ScreenAuditWord into `words`. Off the timed path: nothing here runs unless
// the audit is on, and it changes no result.
template <class Metric, int KC, bool kKnn>
__device__ __noinline__ void auditTile(unsigned long long *words, uint32_t taddr, const Metric &m,
                                       const float *sA, const float *raw, const float *centre,
                                       int myRow, bool rowValid, int myComp, int firstCol, int n,
                                       const int *cOrig, const int *cComp, bool useComp,
                                       float margin) {
  unsigned long long pairs = 0, violations = 0;
  float minSlack = INFINITY, maxGap = -INFINITY, maxAbs = -INFINITY, exactAbs = -INFINITY,
        exactRel = -INFINITY;
  float a[KC], x[KC];
  double ni = 0.0;
#pragma unroll
  for (int k = 0; k < KC; ++k) {
    a[k] = sA[k * kTile + myRow];
    x[k] = a[k] - centre[k];
    ni += (double)x[k] * (double)x[k];
  }
#pragma unroll 1
  for (int chunk = 0; chunk < 4; ++chunk) {
    float v[32];
    tmemLoad32(taddr + chunk * 32, v);
#pragma unroll 1
    for (int c = 0; c < 32; ++c) {
      const int jj = chunk * 32 + c;
      if (!rowValid || firstCol + jj >= n || cOrig[jj] < 0)
        continue;
      if (!kKnn && (useComp ? cComp[jj] : cOrig[jj]) == myComp)
        continue;
      typename Metric::Acc acc = m.init();
      double s, s64, norms;
      if constexpr (std::is_same<Metric, CosineMetric>::value) {
        // The screened value bounds the distance itself; the margin is
        // absolute (norms = 1).
        double dot = 0.0, na = 0.0, nb = 0.0;
#pragma unroll
        for (int k = 0; k < KC; ++k) {
          const float b = raw[k * kTile + jj];
          acc = m.accumulate(acc, a[k], b);
          dot = fma((double)a[k], (double)b, dot);
          na = fma((double)a[k], (double)a[k], na);
          nb = fma((double)b, (double)b, nb);
        }
        s = (double)m.finalize(acc);
        s64 = na * nb > 0.0 ? 1.0 - dot / sqrt(na * nb) : 1.0;
        norms = 1.0;
      } else {
        double nj = 0.0;
        s64 = 0.0;
#pragma unroll
        for (int k = 0; k < KC; ++k) {
          const float b = raw[k * kTile + jj];
          acc = m.accumulate(acc, a[k], b);
          const double diff = (double)a[k] - (double)b;
          s64 = fma(diff, diff, s64);
          const float y = b - centre[k];
          nj = fma((double)y, (double)y, nj);
        }
        s = (double)acc;
        norms = ni + nj;
      }
      const double dp = (double)v[c];
      ++pairs;
      if (dp > s + 0x1p-70)
        ++violations;
      // The relative margin is the guarantee where it exceeds the absolute
      // 2^-70 (below it, flushed and underflowed products are covered by
      // the absolute term alone, and D' <= s + 2^-70 is what counts).
      if ((double)margin * norms > 0x1p-70) {
        minSlack = fminf(minSlack, (float)((s - dp) / ((double)margin * norms)));
        maxGap = fmaxf(maxGap, (float)((s64 - dp) / norms));
      }
      maxAbs = fmaxf(maxAbs, (float)(s64 - dp));
      exactAbs = fmaxf(exactAbs, (float)fabs(s - s64));
      if (s64 > 0.0)
        exactRel = fmaxf(exactRel, (float)(fabs(s - s64) / s64));
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off /= 2) {
    pairs += __shfl_xor_sync(0xffffffffu, pairs, off);
    violations += __shfl_xor_sync(0xffffffffu, violations, off);
    minSlack = fminf(minSlack, __shfl_xor_sync(0xffffffffu, minSlack, off));
    maxGap = fmaxf(maxGap, __shfl_xor_sync(0xffffffffu, maxGap, off));
    maxAbs = fmaxf(maxAbs, __shfl_xor_sync(0xffffffffu, maxAbs, off));
    exactAbs = fmaxf(exactAbs, __shfl_xor_sync(0xffffffffu, exactAbs, off));
    exactRel = fmaxf(exactRel, __shfl_xor_sync(0xffffffffu, exactRel, off));
  }
  if ((threadIdx.x & 31) == 0 && pairs > 0) {
    atomicAdd(words + kAuditPairs, pairs);
    if (violations)
      atomicAdd(words + kAuditViolations, violations);
    if (minSlack < INFINITY)
      atomicMax(words + kAuditMinSlack, (unsigned long long)(~orderedBits(minSlack)));
    if (maxGap > -INFINITY)
      atomicMax(words + kAuditMaxBoundGap, (unsigned long long)orderedBits(maxGap));
    atomicMax(words + kAuditMaxBoundAbs, (unsigned long long)orderedBits(maxAbs));
    atomicMax(words + kAuditMaxExactAbs, (unsigned long long)orderedBits(exactAbs));
    if (exactRel > -INFINITY)
      atomicMax(words + kAuditMaxExactRel, (unsigned long long)orderedBits(exactRel));
  }
}

// kAudit: the audited variant (launched only while cuhc_set_screen_audit is
// on), so that the audit costs the normal kernel nothing.
template <class Metric, class Weight, int KC, bool kKnn, bool kAudit>
__global__ void __launch_bounds__(kThreads, 2)
    screenKernel(PassParams p, Metric m, Weight w, float margin, int stages, int leadArg) {
  using L = ScreenLayout<KC>;
  const L layout{stages};
  constexpr int kPad = L::kPad;
  constexpr uint32_t kSbo = kPad * 32;
  constexpr int R = screenSlots(KC);
  const int S = stages;
  const int lead = leadArg;
  extern __shared__ __align__(128) float dyn[];
  __shared__ PassState sh;
  __shared__ ScreenSync ss;
  // Bounding box of each consumer warp's valid rows (+inf/-inf when none).
  __shared__ float groupLow[4 * KC], groupHigh[4 * KC];
  // k-NN: the largest centred squared norm of each consumer warp's valid rows.
  __shared__ float groupNorm[4];
  float *sA = dyn + layout.sA();
  float *rawBase = dyn + layout.raw();
  int *metaBase = reinterpret_cast<int *>(dyn + layout.meta());
  float *opA = dyn + layout.opA(), *opB = dyn + layout.opB();
  float *rowLow = dyn + layout.box(), *rowHigh = rowLow + KC, *centre = rowHigh + KC;
  unsigned long long *lists = reinterpret_cast<unsigned long long *>(dyn + layout.lists());

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool consumer = tid < kTile;
  const bool producer = tid == kProducerWarp * 32, mmaThread = tid == kMmaWarp * 32;
  const int I = p.tileOrder ? p.tileOrder[blockIdx.x] : (int)blockIdx.x;
  const int firstRow = I * kTile;
  const int leaf = p.leafOfTile[I];
  const int rowPure = (!kKnn && p.nodePure) ? p.nodePure[leaf] : -1;
  const float rowMinValue = p.nodeMinValue ? p.nodeMinValue[leaf] : 0.0f;
  const float slack = 1.0f - boxSlack(p.d);
  const bool useComp = !kKnn && p.component != nullptr;
  const bool useValue = !kKnn && w.value != nullptr;
  const float scale = 1.0f - margin;
  constexpr bool kCos = std::is_same<Metric, CosineMetric>::value;
  // Cosine: 1 - e rounded down to TF32 (10 mantissa bits; the FP32 rounding of
  // 1 - e is far inside the margin's factor two).
  const float cosC = __uint_as_float(__float_as_uint(1.0f - margin) & ~0x1fffu);

  // Consumer row state (thread = row).
  const int myRow = tid & (kTile - 1);
  const int myPos = firstRow + myRow;
  const bool myValid = consumer && myPos < p.n && p.order[myPos] >= 0; // not a padding slot
  const int myComp = myValid ? (p.component ? p.component[myPos] : p.order[myPos]) : -2;
  const float myVal = myValid ? w.load(myPos) : 0.0f;
  // A seed is a real edge of the row; a settled seed is its answer already
  // (written before the pass): the row neither searches nor writes.
  const unsigned long long mySeed =
      (!kKnn && myValid && p.seedKey) ? p.seedKey[myPos] : kEmptyKey;
  const bool settled = mySeed != kEmptyKey && (mySeed & kSettledKey) != 0;
  const bool mySearch = myValid && !settled;
  unsigned int *compSlot = (!kKnn && mySearch && p.compBest) ? p.compBest + myComp : nullptr;

  if (kKnn)
    for (int i = tid; i < kTile * p.k; i += kThreads) {
      lists[i] = kEmptyListKey;
    }
  for (int f = tid; f < KC; f += kThreads) {
    const bool real = f < p.d;
    const float lo = real ? p.nodeLow[(size_t)leaf * p.d + f] : 0.0f;
    const float hi = real ? p.nodeHigh[(size_t)leaf * p.d + f] : 0.0f;
    rowLow[f] = lo;
    rowHigh[f] = hi;
    centre[f] = real ? 0.5f * (lo + hi) : 0.0f;
  }
  copyChunk(sA, p.tiled + (size_t)I * L::rawFloats, KC * kTile);
  if (warp == 0) {
    tmemAlloc(&ss.tmemBase, 256);
    tmemRelinquish();
  }
  const bool wantOneHot = !kKnn && useComp && !p.singletons;
  int *rowComps = metaBase; // ring slot 0 is free until the first copy
  if (consumer && wantOneHot)
    rowComps[myRow] = mySearch ? myComp : -1;
  if (tid == 0) {
    // Arrival counts: rawFull takes the producer's expect-tx (or sentinel)
    // arrival, rawEmpty one per consumer warp, mmaFull the MMA commit + the
    // MMA thread's release of slotTile, tmemEmpty one per consumer warp,
    // opBReady one per builder warp.
    for (int s = 0; s < S; ++s) {
      mbarrierInit(&ss.rawFull[s], 1);
      mbarrierInit(&ss.rawEmpty[s], 4);
    }
    for (int s = 0; s < 2; ++s) {
      mbarrierInit(&ss.mmaFull[s], 2);
      mbarrierInit(&ss.tmemEmpty[s], 4);
      mbarrierInit(&ss.opBReady[s], kBuilderWarps);
    }
    fenceBarrierInit();
    ss.failed = 0;
    ss.oneHot = 0;
    ss.rowSetCount = 0;
    sh.frontLen = 0;
    sh.overflow = 0;
    const int root = p.rootOfTile ? p.rootOfTile[I] : 0;
    const int rootPure = (!kKnn && p.nodePure) ? p.nodePure[root] : -1;
    if (!(rowPure >= 0 && rootPure == rowPure)) {
      sh.frontNode[0] = root;
      sh.frontLen = 1;
    }
  }
  __syncthreads();
  if (wantOneHot && tid == 0) {
    // Distinct components of the row tile, up to R.
    int count = 0;
    bool ok = true;
    for (int i = 0; i < kTile && ok; ++i) {
      const int c = rowComps[i];
      if (c < 0)
        continue;
      bool found = false;
      for (int q = 0; q < count; ++q)
        found |= ss.rowSet[q] == c;
      if (!found) {
        if (count == R)
          ok = false;
        else
          ss.rowSet[count++] = c;
      }
    }
    ss.rowSetCount = count;
    ss.oneHot = ok ? 1 : 0;
  }
  __syncthreads();
  tcgenFenceAfter();
  const uint32_t tmem = ss.tmemBase;
  const bool oneHot = ss.oneHot != 0;
  float myNorm = 0.0f; // k-NN: the row's centred squared norm
  if (consumer) {
    if constexpr (kCos)
      buildRowOperandCosine<KC>(sA, myRow, mySearch, myComp, ss, opA);
    else
      buildRowOperand<KC>(sA, centre, scale, myRow, mySearch, myComp, ss, opA);
    if (kKnn) {
      float nrm = 0.0f;
#pragma unroll
      for (int k = 0; k < KC; ++k) {
        const float x = sA[k * kTile + myRow] - centre[k];
        nrm = fmaf(x, x, nrm);
      }
      myNorm = myValid ? nrm : 0.0f;
      float mx = myNorm;
#pragma unroll
      for (int off = 16; off > 0; off /= 2)
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, off));
      if (lane == 0)
        groupNorm[warp] = mx;
    }
#pragma unroll
    for (int k = 0; k < KC; ++k) {
      float lo = mySearch ? sA[k * kTile + myRow] : INFINITY;
      float hi = mySearch ? sA[k * kTile + myRow] : -INFINITY;
#pragma unroll
      for (int off = 16; off > 0; off /= 2) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, off));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, off));
      }
      if (lane == 0) {
        groupLow[warp * KC + k] = lo;
        groupHigh[warp * KC + k] = hi;
      }
    }
  }
  fenceProxyAsync();

  // Row threshold: sets F (the row's filter bound) and returns the row's
  // threshold for the block maximum (-inf for rows that can gain nothing).
  unsigned long long rowBest = settled ? kEmptyKey : mySeed;
  int tie = 0; // k-NN: a point outside the row's list ties its k-th value
  float F = -INFINITY;
  float rowThr = INFINITY; // the row's weight threshold at the last refresh
  auto refresh = [&](unsigned int cb) -> float {
    float thr;
    if (kKnn) {
      thr = listKeyValue(lists[myRow * p.k + p.k - 1]);
      F = mySearch ? m.screenBound(thr) : -INFINITY;
    } else {
      thr = rowBest == kEmptyKey ? INFINITY : keyWeight(rowBest);
      if (compSlot) {
        if (rowBest != kEmptyKey && floatBits(thr) < cb)
          cb = min(cb, atomicMin(compSlot, floatBits(thr)));
        thr = fminf(thr, bitsFloat(cb));
      }
      // A proposed radius caps the threshold after the component exchange
      // (only real edge weights go into compBest); negative: settled row.
      if (mySearch && p.radius)
        thr = fminf(thr, p.radius[myPos]);
      F = (mySearch && thr >= 0.0f && w.feasible(thr, myVal))
              ? m.screenBound(w.distBound(thr, myVal))
              : -INFINITY;
    }
    rowThr = thr;
    return F == -INFINITY ? -INFINITY : thr;
  };
  // Publishes the warp's largest threshold (for the block's candidate cut),
  // each row's F and the warp's largest F (for the tile tests).
  auto publish = [&](float t) {
    float f = F;
#pragma unroll
    for (int off = 16; off > 0; off /= 2) {
      t = fmaxf(t, __shfl_xor_sync(0xffffffffu, t, off));
      f = fmaxf(f, __shfl_xor_sync(0xffffffffu, f, off));
    }
    ss.rowF[myRow] = F;
    if (lane == 0) {
      ss.warpThr[warp] = t;
      ss.groupF[warp] = f;
    }
  };
  if (consumer)
    publish(refresh(compSlot ? __ldcg(compSlot) : 0xffffffffu));
  __syncthreads();
  if (tid == 0)
    sh.thrTile = fmaxf(fmaxf(ss.warpThr[0], ss.warpThr[1]), fmaxf(ss.warpThr[2], ss.warpThr[3]));
  __syncthreads();

  const uint32_t idesc = umma_idesc_tf32(128, 128);
  const bool maskPass = useComp && !p.singletons;
  const uint32_t metaBytes =
      (uint32_t)(kTile * sizeof(int)) * (p.packedMeta ? 3 : 1 + useComp + useValue);
  const uint32_t tileBytes = (uint32_t)(L::rawFloats * sizeof(float));
  int t = 0;      // ordinal of tiles and sentinels through the rings (all threads agree)
  int tSlot = 0, tPhase = 0; // t % S and the parity of t / S
  auto nextOrdinal = [&]() {
    ++t;
    if (++tSlot == S) {
      tSlot = 0;
      tPhase ^= 1;
    }
  };
  int issued = 0; // producer: ordinals issued
  int iSlot = 0; // producer: issued % S
  int qSlot = 0, qPhase = 0; // producer: (issued - lead) % S and its parity
  int lastCommit = -1;
  unsigned long long prefiltered = 0; // candidate tiles no row needed (per thread)
  unsigned long long computed = 0;
  bool selfPending = kKnn || rowPure < 0;
  bool overflow = false;
  bool dirty = false;                          // consumer: row filter may have tightened
  unsigned long long rechecks = 0, slowRows = 0; // consumer counters

  const float pruneScale = (1.0f - boxSlack(p.d)) * (1.0f - boxSlack(p.d));
  // Whether any row of the tile can still gain from column tile `entry`:
  // its point-to-box squared lower bound (scaled by the box slack) at most
  // the row's published filter bound. One thread per candidate: the box in
  // registers (features past d are zero on both sides and add nothing), rows
  // and bounds read as shared-memory broadcasts, stopping at the first row
  // that needs the tile. Each warp's 32 rows are first tested as a group:
  // the box-to-box bound against the group's largest F. Rounding is
  // monotone, so the group bound never exceeds any member row's bound and
  // a group that fails holds no row that passes.
  auto rowsNeed = [&](int entry) -> bool {
    const int leafJ = p.leafOfTile[entry & ~kPureColumnTile];
    const float *lo = p.nodeLow + (size_t)leafJ * p.d, *hi = p.nodeHigh + (size_t)leafJ * p.d;
    float blo[KC], bhi[KC];
#pragma unroll
    for (int k = 0; k < KC; ++k) {
      blo[k] = k < p.d ? __ldg(lo + k) : 0.0f;
      bhi[k] = k < p.d ? __ldg(hi + k) : 0.0f;
    }
    for (int g = 0; g < 4; ++g) {
      const float gF = ((volatile float *)ss.groupF)[g];
      if (!(gF >= 0.0f))
        continue; // no row of the group gains anything
      float b2 = 0.0f;
#pragma unroll
      for (int k = 0; k < KC; ++k) {
        const float gap = fmaxf(0.0f, fmaxf(blo[k] - groupHigh[g * KC + k],
                                            groupLow[g * KC + k] - bhi[k]));
        b2 = fmaf(gap, gap, b2);
      }
      if (b2 * pruneScale > gF)
        continue;
      for (int r = 32 * g; r < 32 * g + 32; ++r) {
        const float F = ((volatile float *)ss.rowF)[r];
        if (!(F >= 0.0f))
          continue; // a row that gains nothing
        float s2 = 0.0f;
#pragma unroll
        for (int k = 0; k < KC; ++k) {
          const float x = sA[k * kTile + r];
          const float gap = fmaxf(0.0f, fmaxf(blo[k] - x, x - bhi[k]));
          s2 = fmaf(gap, gap, s2);
        }
        if (s2 * pruneScale <= F)
          return true;
      }
    }
    return false;
  };
  int batch = 0;
  while (true) {
    if (warp == 0)
      collectCandidates(p, m, w, sh, rowLow, rowHigh, I, rowPure, rowMinValue, slack);
    __syncthreads();
    const int len = sh.listLen;
    if (sh.overflow) {
      overflow = true;
      break;
    }
    if (len == 0 && sh.frontLen == 0 && !selfPending)
      break;
    if (p.prune && len > 1)
      sortCandidates(sh, len);
    __syncthreads();

    // Phases of the batch: the producer issues phaseLimit tiles (kFirstPhase,
    // then eight times more each phase) and a sentinel; between phases every
    // warp tests the remaining candidates against the rows' current bounds.
    int cursor = 0, phaseLimit = kFirstPhase;
    for (int phase = 0;; ++phase) {
    if (p.prune && (batch > 0 || phase > 0)) {
      for (int c = cursor + tid; c < len; c += kThreads)
        if (sh.listLb[c] < INFINITY && !rowsNeed(sh.listTile[c])) {
          sh.listLb[c] = INFINITY;
          ++prefiltered;
        }
      __syncthreads();
    }

    if (warp == kProducerWarp) {
      // ---- producer: the warp picks candidate tiles, lane 0 issues the
      // bulk copies; one ordinal per step until the phase's sentinel ----
      int phaseIssued = 0;
      while (true) {
        // Every consumer warp has finished ordinal issued - lead (and so the
        // slot's previous ordinal, issued - stages). Every ordinal, sentinels
        // included, passes through rawEmpty once, so the parity follows the
        // ordinal, and the slot's next use is not issued yet.
        if (issued >= lead) {
          if (!__shfl_sync(0xffffffffu, screenWait(&ss.rawEmpty[qSlot], qPhase, ss), 0))
            break;
          if (++qSlot == S) {
            qSlot = 0;
            qPhase ^= 1;
          }
        }
        const int r = iSlot;
        int entry = -1;
        if (selfPending) {
          entry = I;
          selfPending = false;
        } else if (phaseIssued < phaseLimit) {
          // The next entry whose bound is within the block threshold, 32
          // entries per step (entries the tile test dropped hold +inf).
          const float thr =
              __shfl_sync(0xffffffffu, lane == 0 ? *(volatile float *)&sh.thrTile : 0.0f, 0);
          while (cursor < len) {
            const int c = cursor + lane;
            const unsigned hit = __ballot_sync(0xffffffffu, c < len && !(sh.listLb[c] > thr));
            if (hit) {
              cursor += __ffs(hit) - 1;
              entry = sh.listTile[cursor++];
              break;
            }
            cursor += 32;
          }
          cursor = min(cursor, len);
        }
        if (entry >= 0)
          ++phaseIssued;
        if (lane == 0) {
          ss.rawTile[r] = entry;
          if (entry < 0) {
            mbarrierArrive(&ss.rawFull[r], 1);
          } else {
            const int J = entry & ~kPureColumnTile;
            int *meta = metaBase + r * L::metaInts;
            mbarrierArriveExpectTx(&ss.rawFull[r], tileBytes + metaBytes);
            bulkCopyToShared(rawBase + r * L::rawFloats, p.tiled + (size_t)J * L::rawFloats,
                             tileBytes, &ss.rawFull[r]);
            if (p.packedMeta) {
              bulkCopyToShared(meta, p.packedMeta + (size_t)J * 3 * kTile, metaBytes,
                               &ss.rawFull[r]);
            } else {
              bulkCopyToShared(meta, p.order + (size_t)J * kTile, kTile * sizeof(int),
                               &ss.rawFull[r]);
              if (useComp)
                bulkCopyToShared(meta + kTile, p.component + (size_t)J * kTile,
                                 kTile * sizeof(int), &ss.rawFull[r]);
              if (useValue)
                bulkCopyToShared(meta + 2 * kTile, w.value + (size_t)J * kTile,
                                 kTile * sizeof(float), &ss.rawFull[r]);
            }
          }
        }
        ++issued;
        if (++iSlot == S)
          iSlot = 0;
        if (entry < 0)
          break;
      }
    } else if (warp == kMmaWarp) {
      // ---- MMA warp: lane 0 issues the MMAs, the warp runs in step ----
      while (true) {
        const int s = t & 1;
        // Every consumer warp has read ordinal t - 2: accumulator s is free.
        bool ok = __shfl_sync(0xffffffffu, screenWait(&ss.tmemEmpty[s], ((t >> 1) & 1) ^ 1, ss), 0);
        // The builders finished ordinal t: its column operand, or (a
        // sentinel) their pass through it, after the producer staged it. Waited
        // for the sentinel too: its mmaFull arrival below completes that
        // barrier's phase of ordinal t, and it must not do so before every
        // builder has waited on the phase of ordinal t - 2 -- a parity wait two
        // phases behind would see its parity again and wait for a phase that
        // never comes.
        if (ok)
          ok = screenWait(&ss.opBReady[s], (t >> 1) & 1, ss);
        ok = __shfl_sync(0xffffffffu, ok, 0);
        const int entry = ok ? ss.rawTile[tSlot] : -1;
        ok = ok && entry >= 0;
        if (lane == 0) {
          if (ok) {
            tcgenFenceAfter();
            const float *b = opB + (size_t)s * kTile * kPad;
#pragma unroll
            for (int ks = 0; ks < kPad / 8; ++ks)
              mmaTf32(tmem + (uint32_t)(s * kTile), umma_smem_desc(opA + 64 * ks, 128, kSbo),
                      umma_smem_desc(b + 64 * ks, 128, kSbo), idesc, ks > 0);
            mmaCommit(&ss.mmaFull[s]);
            lastCommit = t;
            ss.slotTile[s] = entry;
            mbarrierArrive(&ss.mmaFull[s], 1);
          } else {
            ss.slotTile[s] = -1; // the batch's end (or a failed wait) goes on to the consumers
            mbarrierArrive(&ss.mmaFull[s], 2);
          }
        }
        nextOrdinal();
        if (!ok)
          break;
      }
    } else if (!consumer) {
      // ---- builders: warps 4..5, columns j and j + 64 ----
      const int j = tid - kTile;
      float cen[KC];
#pragma unroll
      for (int k = 0; k < KC; ++k)
        cen[k] = centre[k];
      while (true) {
        const int s = t & 1;
        // The operand buffer of slot s is free once the MMA of ordinal t - 2
        // has completed (the consumers may still be reading its result).
        bool ok = screenWait(&ss.mmaFull[s], ((t >> 1) & 1) ^ 1, ss);
        const int r = tSlot;
        ok = screenWait(&ss.rawFull[r], tPhase, ss) && ok;
        const int entry = __shfl_sync(0xffffffffu, ok ? ss.rawTile[r] : -1, 0);
        if (entry >= 0) {
          const float *raw = rawBase + r * L::rawFloats;
          const int *comp = metaBase + r * L::metaInts + kTile;
          float *b = opB + (size_t)s * kTile * kPad;
#pragma unroll
          for (int q = j; q < kTile; q += kBuilderThreads)
            if constexpr (kCos)
              buildColumnOperandCosine<KC>(raw, comp, cosC, q, oneHot, ss, b);
            else
              buildColumnOperand<KC>(raw, comp, cen, scale, q, oneHot, ss, b);
        }
        fenceProxyAsync();
        __syncwarp();
        if (lane == 0)
          mbarrierArrive(&ss.opBReady[s], 1);
        nextOrdinal();
        if (entry < 0)
          break;
      }
    } else {
      // ---- consumers: warps 0..3, row myRow = tensor-memory lane ----
      unsigned long long *list = lists + myRow * p.k;
      while (true) {
        const int s = t & 1;
        const bool ok = screenWait(&ss.mmaFull[s], (t >> 1) & 1, ss);
        tcgenFenceAfter();
        const int entry = __shfl_sync(0xffffffffu, ok ? ss.slotTile[s] : -1, 0);
        const int r = tSlot;
        bool thrChanged = false;
        if (entry >= 0) {
          const int J = entry & ~kPureColumnTile;
          const bool colPure = (entry & kPureColumnTile) != 0;
          const float *raw = rawBase + r * L::rawFloats;
          const int *cOrig = metaBase + r * L::metaInts;
          const int *cComp = cOrig + kTile;
          const float *cVal = reinterpret_cast<const float *>(cOrig + 2 * kTile);
          const bool mask = maskPass && !oneHot && !(rowPure >= 0 && colPure);
          const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(s * kTile);
          // Each half: two 32-column chunk loads in flight, the row minimum of
          // D' over them (own component excluded when masking, two chains per
          // chunk), and -- only when some row of the warp has a value within
          // its bound -- the candidate bits of both chunks, built from the
          // same registers (no second read of tensor memory).
          float Fs = F + kScreenAbsSlack;
          if constexpr (std::is_same<Weight, WardWeight>::value) {
            // Ward: F assumes the lightest partner (size 1); the column tile's
            // smallest cluster size s_min tightens it, since 2 si sj / (si + sj)
            // grows with sj: a pair weighs <= thr only if its squared distance
            // is <= thr (1/si + 1/s_min) / 2 (rounded up, as distBound).
            float sMin = INFINITY;
#pragma unroll
            for (int c = lane; c < kTile; c += 32)
              if (J * kTile + c < p.n && cOrig[c] >= 0)
                sMin = fminf(sMin, cVal[c]);
#pragma unroll
            for (int off = 16; off > 0; off /= 2)
              sMin = fminf(sMin, __shfl_xor_sync(0xffffffffu, sMin, off));
            if (F > -INFINITY && rowThr < INFINITY && sMin < INFINITY)
              Fs = fminf(Fs, m.screenBound(__fmul_ru(
                                 rowThr, (1.0f / myVal + 1.0f / sMin) * 0.5f * 1.00001f)) +
                                 kScreenAbsSlack);
          }
          if (kKnn && J == I && p.k <= kTile) {
            // delta: 1.5 e (|x|^2 + |y|^2) bounds s - D' (the margin e is twice
            // the error bound); twice that, with the tile's largest norm.
            const float normMax = fmaxf(fmaxf(groupNorm[0], groupNorm[1]),
                                        fmaxf(groupNorm[2], groupNorm[3]));
            const float delta =
                (kCos ? 2.0f * margin : 2.02f * margin * (myNorm + normMax)) + 0x1p-60f;
            Fs = fminf(Fs, selfTileBound(taddr, cOrig, J * kTile, p.n, p.k, delta) +
                               kScreenAbsSlack);
          }
          uint32_t cand[4];
#pragma unroll
          for (int half = 0; half < 2; ++half) {
            uint32_t a[32], b[32];
            tmemLoad32Async(taddr + half * 64, a);
            tmemLoad32Async(taddr + half * 64 + 32, b);
            tmemWaitLoads(a);
            tmemHold(b);
            float pa0 = INFINITY, pa1 = INFINITY, pb0 = INFINITY, pb1 = INFINITY;
            if (mask) {
#pragma unroll
              for (int q = 0; q < 16; ++q) {
                const uint32_t *src = q < 8 ? a : b;
                const int c = (q & 7) * 4;
                const int4 cc = reinterpret_cast<const int4 *>(cComp)[half * 16 + q];
                float &part = q < 8 ? ((q & 1) ? pa1 : pa0) : ((q & 1) ? pb1 : pb0);
                part = min3(part, cc.x != myComp ? __uint_as_float(src[c]) : INFINITY,
                            cc.y != myComp ? __uint_as_float(src[c + 1]) : INFINITY);
                part = min3(part, cc.z != myComp ? __uint_as_float(src[c + 2]) : INFINITY,
                            cc.w != myComp ? __uint_as_float(src[c + 3]) : INFINITY);
              }
            } else {
#pragma unroll
              for (int c = 0; c < 32; c += 4) {
                pa0 = min3(pa0, __uint_as_float(a[c]), __uint_as_float(a[c + 1]));
                pa1 = min3(pa1, __uint_as_float(a[c + 2]), __uint_as_float(a[c + 3]));
                pb0 = min3(pb0, __uint_as_float(b[c]), __uint_as_float(b[c + 1]));
                pb1 = min3(pb1, __uint_as_float(b[c + 2]), __uint_as_float(b[c + 3]));
              }
            }
            const bool wantA = mySearch && fminf(pa0, pa1) <= Fs;
            const bool wantB = mySearch && fminf(pb0, pb1) <= Fs;
            uint32_t ca = 0, cb = 0;
            if (__any_sync(0xffffffffu, wantA || wantB)) {
#pragma unroll
              for (int c = 0; c < 32; ++c) {
                ca |= (__uint_as_float(a[c]) <= Fs ? 1u : 0u) << c;
                cb |= (__uint_as_float(b[c]) <= Fs ? 1u : 0u) << c;
              }
              ca = wantA ? ca : 0u;
              cb = wantB ? cb : 0u;
            }
            cand[2 * half] = ca;
            cand[2 * half + 1] = cb;
          }
          if (kAudit)
            auditTile<Metric, KC, kKnn>(p.screenAudit, taddr, m, sA, raw, centre, myRow, myValid,
                                        myComp, J * kTile, p.n, cOrig, cComp, useComp, margin);
          // Done with accumulator s: the MMA of ordinal t + 2 may overwrite it
          // while this warp rechecks.
          tcgenFenceBefore();
          __syncwarp();
          if (lane == 0)
            mbarrierArrive(&ss.tmemEmpty[s], 1);
          uint32_t c0 = cand[0], c1 = cand[1], c2 = cand[2], c3 = cand[3];
          if (__any_sync(0xffffffffu, (c0 | c1 | c2 | c3) != 0)) {
            slowRows += (c0 | c1 | c2 | c3) != 0;
            // The candidates of the row, chunk by chunk: c0 holds the current
            // chunk (columns base .. base + 31) and the others shift down.
            int base = 0;
            // k-NN: the row's k-th value, reloaded only after an insertion.
            float rowKth = kKnn && mySearch ? listKeyValue(list[p.k - 1]) : 0.0f;
            while (c0 | c1 | c2 | c3) {
              if (c0 == 0) {
                c0 = c1;
                c1 = c2;
                c2 = c3;
                c3 = 0;
                base += 32;
                continue;
              }
              const int jj = base + __ffs(c0) - 1;
              c0 &= c0 - 1;
              if (J * kTile + jj >= p.n || cOrig[jj] < 0)
                continue; // beyond the points, or a padding slot
              if (!kKnn && (useComp ? cComp[jj] : cOrig[jj]) == myComp)
                continue;
              // The reference's exact FP32 distance (zero-padded features add 0).
              typename Metric::Acc acc = m.init();
#pragma unroll
              for (int k = 0; k < KC; ++k)
                acc = m.accumulate(acc, sA[k * kTile + myRow], raw[k * kTile + jj]);
              ++rechecks;
              if (kKnn) {
                const float value = J * kTile + jj == myPos ? 0.0f : fmaxf(m.finalize(acc), 0.0f);
                // Offer to the row's list (the k-th value kept in a register):
                // a value below the k-th enters, and the boundary-tie flag
                // follows knnOffer (passes.cuh): an insertion evicts the old
                // k-th, which ties the new k-th when they are equal; a value
                // equal to the k-th that stays out ties it.
                if (value < rowKth) {
                  const float c = value > 0.0f ? value : 0.0f; // +0 for -0: bits order like values
                  insertListKey(list, p.k,
                                ((unsigned long long)__float_as_uint(c) << 32) |
                                    (uint32_t)(J * kTile + jj));
                  const float old = rowKth;
                  rowKth = listKeyValue(list[p.k - 1]);
                  tie = (old < INFINITY && rowKth == old) ? 1 : 0;
                  Fs = m.screenBound(rowKth) + kScreenAbsSlack;
                  dirty = true;
                } else if (value == rowKth) {
                  tie = 1;
                }
              } else {
                const float weight = w.weight(m.finalize(acc), myVal, useValue ? cVal[jj] : 0.0f);
                if (weight < INFINITY) {
                  const unsigned long long key = packKey(weight, (uint32_t)cOrig[jj]);
                  if (key < rowBest) {
                    rowBest = key;
                    dirty = true;
                  }
                }
              }
            }
          }
          // The row's filter changes only through its own exact path or the
          // component's best (found by other blocks): refresh then, and every
          // eighth tile for the latter.
          if (__any_sync(0xffffffffu, dirty) || (computed & 7) == 7) {
            publish(refresh(compSlot ? __ldcg(compSlot) : 0xffffffffu));
            dirty = false;
            thrChanged = true;
          }
          ++computed;
        } else {
          tcgenFenceBefore();
          __syncwarp();
          if (lane == 0)
            mbarrierArrive(&ss.tmemEmpty[s], 1);
        }
        __syncwarp();
        if (lane == 0) {
          // This warp is done with ring slot r (every ordinal, sentinels
          // included, passes through rawEmpty and tmemEmpty once).
          mbarrierArrive(&ss.rawEmpty[r], 1);
          if (thrChanged)
            *(volatile float *)&sh.thrTile = fmaxf(fmaxf(ss.warpThr[0], ss.warpThr[1]),
                                                   fmaxf(ss.warpThr[2], ss.warpThr[3]));
        }
        nextOrdinal();
        if (entry < 0)
          break;
      }
    }
    if (warp == kProducerWarp && lane == 0) {
      ss.cursor = cursor;
      ss.batchDone = cursor >= len ? 1 : 0;
    }
    __syncthreads();
    // The producer issued the row tile itself first in the first phase; every
    // thread forgets it here so that the loop's exit stays uniform.
    selfPending = false;
    cursor = ss.cursor;
    if (ss.failed || ss.batchDone)
      break;
    phaseLimit *= 8;
    } // phases
    ++batch;
    if (ss.failed)
      break;
    if (sh.frontLen == 0)
      break;
  }

  // Nothing may land in shared or tensor memory after the block leaves: on a
  // failure the producer waits (bounded) for its copies (each slot's last
  // use) and the MMA thread for its last MMAs.
  if (producer && ss.failed)
    for (int o = max(0, issued - S); o < issued; ++o)
      mbarrierWait(&ss.rawFull[o % S], (o / S) & 1);
  if (mmaThread && ss.failed && lastCommit >= 0)
    mbarrierWait(&ss.mmaFull[lastCommit & 1], (lastCommit >> 1) & 1);
  if (consumer && myPos < p.n) {
    if (kKnn) {
      const int rank = myValid ? (p.coreRank ? p.coreRank[myPos] : p.k) : 0;
      p.core[myPos] = rank > 0 ? listKeyValue(lists[myRow * p.k + rank - 1]) : 0.0f;
      if (p.knnPos) {
        for (int e = 0; e < p.k; ++e)
          p.knnPos[(size_t)myPos * p.k + e] = (int)(uint32_t)lists[myRow * p.k + e];
        p.knnTie[myPos] = tie;
      }
    } else if ((!p.radius || p.radius[myPos] >= 0.0f) && !settled) {
      p.nearest[myPos] = rowBest;
    }
  }
  if (consumer && p.screenStats) {
    for (int off = 16; off > 0; off /= 2) {
      rechecks += __shfl_xor_sync(0xffffffffu, rechecks, off);
      slowRows += __shfl_xor_sync(0xffffffffu, slowRows, off);
    }
    if (lane == 0) {
      atomicAdd(p.screenStats + kScreenRechecks, rechecks);
      atomicAdd(p.screenStats + kScreenSlowRows, slowRows);
    }
  }
  if (p.screenStats) {
    for (int off = 16; off > 0; off /= 2)
      prefiltered += __shfl_xor_sync(0xffffffffu, prefiltered, off);
    if (lane == 0 && prefiltered)
      atomicAdd(p.screenStats + kScreenPrefiltered, prefiltered);
  }
  tcgenFenceBefore();
  __syncthreads();
  if (warp == 0) {
    tcgenFenceAfter();
    tmemDealloc(tmem, 256);
  }
  if (tid == 0) {
    if (p.tileWork)
      p.tileWork[I] = (unsigned int)computed;
    if (p.tilesComputed)
      atomicAdd(p.tilesComputed, computed);
    if (p.screenStats && maskPass)
      atomicAdd(p.screenStats + (oneHot ? kScreenIndicatorTiles : kScreenMaskedTiles), computed);
    if ((ss.failed || overflow) && p.error)
      atomicCAS(p.error, 0, overflow ? (int)kErrorTooLarge : (int)kErrorTimeout);
  }
}

// Screen mode set by cuhc_set_screen (0 auto, 1 always where supported,
// 2 never). Results are identical in every mode.
int currentScreenMode();

// Pipeline shape of a screened launch: ring slots and copy lead (0: the
// defaults, the most slots that keep two blocks on an SM and screenLead).
// Set per calling thread by the shape tuner (tunedScreenShape); a shape
// changes time only, never a result.
struct ScreenShape {
  int stages = 0, lead = 0;
};
ScreenShape currentScreenShape();
void setScreenShape(ScreenShape shape);

template <class Metric> struct ScreenSupport {
  static constexpr bool value = false;
};
template <> struct ScreenSupport<EuclideanMetric> {
  static constexpr bool value = true;
};
template <> struct ScreenSupport<SqEuclideanMetric> {
  static constexpr bool value = true;
};
template <> struct ScreenSupport<CosineMetric> {
  static constexpr bool value = true;
};

// Shared memory a block may use on sm_100 (227 KiB), and what each of two
// blocks on one SM may use (228 KiB per SM, 1 KiB of it reserved per block).
// A screened block keeps at least kScreenMinShared so that at most two share
// an SM (their tensor memory, 256 columns each, then always fits).
constexpr size_t kMaxBlockShared = 227 * 1024;
constexpr size_t kTwoBlockShared = 113 * 1024;
constexpr size_t kScreenMinShared = 80 * 1024;

// Static shared memory of a screened block (an upper bound).
constexpr size_t kScreenStaticBytes = sizeof(PassState) + sizeof(ScreenSync) + 2 * 4 * 32 * 4;

inline size_t screenLayoutBytes(int d, int k, int stages) {
  switch (chunkWidthFor(d)) {
  case 4:
    return ScreenLayout<4>{stages}.bytes(k);
  case 8:
    return ScreenLayout<8>{stages}.bytes(k);
  case 16:
    return ScreenLayout<16>{stages}.bytes(k);
  default:
    return ScreenLayout<32>{stages}.bytes(k);
  }
}

// Ring slots of a screened pass: the most that keep two blocks on an SM, or,
// when not even kScreenMinStages does, the most that fit one block; 0 when
// nothing fits.
inline int screenStagesFor(int d, int k) {
  for (const size_t limit : {kTwoBlockShared, kMaxBlockShared})
    for (int stages = kScreenMaxStages; stages >= kScreenMinStages; --stages)
      if (screenLayoutBytes(d, k, stages) + kScreenStaticBytes <= limit)
        return stages;
  return 0;
}

inline size_t screenDynamicBytes(int d, int k, int stages) {
  const size_t bytes = screenLayoutBytes(d, k, stages);
  return bytes + kScreenStaticBytes < kScreenMinShared ? kScreenMinShared - kScreenStaticBytes
                                                       : bytes;
}

// Whether a pass over d features (k-NN rank k, 0 for a nearest pass) can run
// screened: the metric has a screened form, the features fit one chunk of at
// most 32, the block's shared memory fits, and screening is not switched off.
// Callers also check the data's extent (SpatialIndex::screenRangeOk).
template <class Metric> inline bool useScreen(int d, int k) {
  return ScreenSupport<Metric>::value && currentScreenMode() != 2 &&
         chunkWidthFor(d) * numChunksFor(d) <= 32 && screenStagesFor(d, k) > 0;
}

// Launches the screened pass; a negative code when the metric or the
// dimension has no screened form (callers check useScreen first).
template <class Metric, class Weight, bool kKnn>
int launchScreen(const PassParams &p, const Metric &m, const Weight &w, int kc,
                 cudaStream_t stream) {
  if constexpr (!ScreenSupport<Metric>::value) {
    return kErrorInvalidAlgorithm;
  } else {
    if (p.numChunks != 1 || kc != chunkWidthFor(p.d))
      return kErrorInvalidAlgorithm;
    const float margin = std::is_same<Metric, CosineMetric>::value
                             ? screenMarginCosine(p.d, kc)
                             : screenMargin(p.d, kc);
    const int maxStages = screenStagesFor(p.d, kKnn ? p.k : 0);
    if (maxStages == 0)
      return kErrorInvalidAlgorithm;
    const ScreenShape shape = currentScreenShape();
    const int stages =
        shape.stages > 0 ? std::max(kScreenMinStages, std::min(shape.stages, maxStages)) : maxStages;
    const int lead = std::max(1, std::min(stages - 1, shape.lead > 0 ? shape.lead
                                                                     : screenLead(kc)));
    const size_t dynBytes = screenDynamicBytes(p.d, kKnn ? p.k : 0, stages);
    auto misaligned = [](const void *ptr) { return ((uintptr_t)ptr & 15) != 0; };
    if (misaligned(p.tiled) || misaligned(p.order) || misaligned(p.component) ||
        misaligned(w.value) || misaligned(p.packedMeta))
      return (int)cudaErrorMisalignedAddress;
    auto run = [&](auto kernel) {
      const cudaError_t e =
          cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dynBytes);
      if (e != cudaSuccess)
        return (int)e;
      kernel<<<p.numTiles, kThreads, dynBytes, stream>>>(p, m, w, margin, stages, lead);
      noteLaunch();
      return (int)cudaGetLastError();
    };
    auto byWidth = [&](auto audit) {
      constexpr bool kAudit = decltype(audit)::value;
      switch (kc) {
      case 4:
        return run(screenKernel<Metric, Weight, 4, kKnn, kAudit>);
      case 8:
        return run(screenKernel<Metric, Weight, 8, kKnn, kAudit>);
      case 16:
        return run(screenKernel<Metric, Weight, 16, kKnn, kAudit>);
      default:
        return run(screenKernel<Metric, Weight, 32, kKnn, kAudit>);
      }
    };
    return p.screenAudit ? byWidth(std::true_type{}) : byWidth(std::false_type{});
  }
}

} // namespace cuhc
