// The tensor-core screened pass: the same nearest / k-NN passes as
// passes.cuh, with the all-pairs distance work moved to tcgen05 MMAs.
//
// Per row tile the block centres every point on the row tile's box centre c
// and builds TF32 operands (K-major, shared memory) such that one
// accumulation over K = 3d + 4 (padded to 8) gives, in tensor memory,
//   D'(i, j) = (1 - e) n_i + (1 - e) n_j - 2 (xh.yh + xh.yl + xl.yh)
// where x = x_i - c = xh + xl and y = y_j - c = yh + yl are TF32 splits and
// n = |x|^2. The margin e (screenMargin) is twice a rigorous bound of every
// error involved, as a multiple of n_i + n_j: the TF32 splits, the dropped
// xl.yl term, the norms' FP32 rounding, the centring rounding, the tensor
// core's FP32 accumulation (modelled pessimistically: every addition off by
// 2^-22 of the sum of absolute products, four times over), and the
// reference's own FP32 rounding of the exact squared distance s. Hence
// D'(i, j) <= s(i, j) for every pair, and a pair can only pass its row's
// filter bound F (a bound on s) if D'(i, j) <= F. Exactly those pairs are
// recomputed with the reference's FP32 fmaf chain from the raw features, so
// every weight, key and k-th distance is bit-identical to the plain pass.
//
// Roles per column tile: warps 4-7 build the column operand (one column per
// thread), thread 0 issues the MMAs and commits them to an mbarrier, warps
// 0-3 read the accumulator (one row per thread: tensor-memory lane = row),
// take the row minimum of D' and recheck only the rows that have a pair at or
// below the filter bound. Candidate collection, nearest-first order and the
// bulk-copy double buffering are those of passes.cuh.
#pragma once

#include <cmath>

#include "passes.cuh"
#include "umma.cuh"

namespace cuhc {

__host__ __device__ inline int screenK(int d) { return (3 * d + 4 + 7) / 8 * 8; }

// e: see the header comment. Units of n_i + n_j.
inline float screenMargin(int d) {
  const double u22 = std::ldexp(1.0, -22), u24 = std::ldexp(1.0, -24);
  const int K = screenK(d);
  const double mma = 4.0 * (9.0 * K / 8.0) * 2.02 * u22;     // accumulation, four times over
  const double split = 3.0 * u22;                             // TF32 splits, dropped lo*lo
  const double norm = ((d + 1) / 4.0 + 1.25) * u22;           // norms, scaling, their split
  const double centre = u22;                                  // rounding of x - c
  const double reference = 2.01 * (d + 1) * u24 * 1.01;       // the exact fmaf chain itself
  return (float)(2.0 * (mma + split + norm + centre + reference));
}

// Warps 4-7 (column j = tid - 128): TF32 operand row of column j of a staged
// raw tile, centred on c.
__device__ __forceinline__ void buildColumnOperand(const float *raw, const float *centre, int d,
                                                   int kPad, float scale, float *op,
                                                   uint32_t sbo, int j) {
  char *base = reinterpret_cast<char *>(op);
  float n = 0.0f;
  for (int k = 0; k < d; ++k) {
    const float y = raw[k * kTile + j] - centre[k];
    n = fmaf(y, y, n);
    const float hi = toTf32(y), lo = toTf32(y - hi);
    *reinterpret_cast<float *>(base + umma_offset(j, k, sbo)) = -2.0f * hi;
    *reinterpret_cast<float *>(base + umma_offset(j, d + k, sbo)) = -2.0f * lo;
    *reinterpret_cast<float *>(base + umma_offset(j, 2 * d + k, sbo)) = -2.0f * hi;
  }
  const float ns = n * scale;
  const float nh = toTf32(ns), nl = toTf32(ns - nh);
  *reinterpret_cast<float *>(base + umma_offset(j, 3 * d, sbo)) = 1.0f;
  *reinterpret_cast<float *>(base + umma_offset(j, 3 * d + 1, sbo)) = 1.0f;
  *reinterpret_cast<float *>(base + umma_offset(j, 3 * d + 2, sbo)) = nh;
  *reinterpret_cast<float *>(base + umma_offset(j, 3 * d + 3, sbo)) = nl;
  for (int k = 3 * d + 4; k < kPad; ++k)
    *reinterpret_cast<float *>(base + umma_offset(j, k, sbo)) = 0.0f;
}

// Threads 0..127 (row i = tid): the row operand (built once per block).
__device__ __forceinline__ void buildRowOperand(const float *raw, const float *centre, int d,
                                                int kPad, float scale, float *op, uint32_t sbo,
                                                int i) {
  char *base = reinterpret_cast<char *>(op);
  float n = 0.0f;
  for (int k = 0; k < d; ++k) {
    const float x = raw[k * kTile + i] - centre[k];
    n = fmaf(x, x, n);
    const float hi = toTf32(x), lo = toTf32(x - hi);
    *reinterpret_cast<float *>(base + umma_offset(i, k, sbo)) = hi;
    *reinterpret_cast<float *>(base + umma_offset(i, d + k, sbo)) = hi;
    *reinterpret_cast<float *>(base + umma_offset(i, 2 * d + k, sbo)) = lo;
  }
  const float ns = n * scale;
  const float nh = toTf32(ns), nl = toTf32(ns - nh);
  *reinterpret_cast<float *>(base + umma_offset(i, 3 * d, sbo)) = nh;
  *reinterpret_cast<float *>(base + umma_offset(i, 3 * d + 1, sbo)) = nl;
  *reinterpret_cast<float *>(base + umma_offset(i, 3 * d + 2, sbo)) = 1.0f;
  *reinterpret_cast<float *>(base + umma_offset(i, 3 * d + 3, sbo)) = 1.0f;
  for (int k = 3 * d + 4; k < kPad; ++k)
    *reinterpret_cast<float *>(base + umma_offset(i, k, sbo)) = 0.0f;
}

template <class Metric, class Weight, int KC, bool kKnn>
__global__ void __launch_bounds__(kThreads, 2)
    screenKernel(PassParams p, Metric m, Weight w, float margin, int kPad) {
  extern __shared__ __align__(128) float dyn[];
  __shared__ PassState sh;
  __shared__ uint64_t mmaBar;
  __shared__ uint32_t tmemBase;
  float *sA = dyn;
  float *sB[2] = {sA + KC * kTile, sA + 2 * KC * kTile};
  int *metaBase = (int *)(sA + 3 * KC * kTile);
  ColumnMeta meta[2];
  for (int b = 0; b < 2; ++b) {
    meta[b].orig = metaBase + b * 3 * kTile;
    meta[b].comp = metaBase + b * 3 * kTile + kTile;
    meta[b].value = (float *)(metaBase + b * 3 * kTile + 2 * kTile);
  }
  float *opA = (float *)(metaBase + 6 * kTile);
  float *opB = opA + kTile * kPad;
  float *rowLow = opB + kTile * kPad;
  float *rowHigh = rowLow + p.d;
  float *centre = rowHigh + p.d;
  float *lists = centre + p.d;
  const uint32_t sbo = (uint32_t)kPad * 32u;

  const int tid = threadIdx.x, warp = tid >> 5;
  const int I = blockIdx.x;
  const int firstRow = I * kTile;
  const int leaf = p.leafOfTile[I];
  const int rowPure = (!kKnn && p.nodePure) ? p.nodePure[leaf] : -1;
  const float rowMinValue = p.nodeMinValue ? p.nodeMinValue[leaf] : 0.0f;
  const float slack = 1.0f - boxSlack(p.d);
  const bool useComp = !kKnn && p.component != nullptr;
  const bool useValue = !kKnn && w.value != nullptr;
  const size_t tileFloats = (size_t)KC * kTile; // one chunk: d <= 32
  const float scale = 1.0f - margin;

  // Epilogue threads own one row each.
  const int myRow = tid & (kTile - 1);
  const int myPos = firstRow + myRow;
  const bool myValid = myPos < p.n;
  const int myComp = myValid ? (p.component ? p.component[myPos] : p.order[myPos]) : -2;
  const float myVal = myValid ? w.load(myPos) : 0.0f;

  if (tid < kTile)
    sh.rowBest[tid] = kEmptyKey;
  if (kKnn)
    for (int i = tid; i < kTile * p.k; i += kThreads)
      lists[i] = INFINITY;
  for (int f = tid; f < p.d; f += kThreads) {
    rowLow[f] = p.nodeLow[(size_t)leaf * p.d + f];
    rowHigh[f] = p.nodeHigh[(size_t)leaf * p.d + f];
    centre[f] = 0.5f * (rowLow[f] + rowHigh[f]);
  }
  copyChunk(sA, p.tiled + (size_t)I * tileFloats, KC * kTile);
  if (warp == 0) {
    tmemAlloc(&tmemBase, kTile);
    tmemRelinquish();
  }
  if (tid == 0) {
    mbarrierInit(&sh.bar[0], 1);
    mbarrierInit(&sh.bar[1], 1);
    mbarrierInit(&mmaBar, 1);
    fenceBarrierInit();
    sh.frontLen = 0;
    sh.overflow = 0;
    const int rootPure = (!kKnn && p.nodePure) ? p.nodePure[0] : -1;
    if (!(rowPure >= 0 && rootPure == rowPure)) {
      sh.frontNode[0] = 0;
      sh.frontLen = 1;
    }
  }
  if (tid < kTile) {
    const int pos = firstRow + tid;
    const bool valid = pos < p.n;
    meta[0].orig[tid] = valid ? p.order[pos] : -1;
    if (useComp)
      meta[0].comp[tid] = valid ? p.component[pos] : -1;
    if (useValue)
      meta[0].value[tid] = valid ? w.load(pos) : 0.0f;
  }
  __syncthreads();
  tcgenFenceAfter();
  const uint32_t tmem = tmemBase;
  if (tid < kTile)
    buildRowOperand(sA, centre, p.d, kPad, scale, opA, sbo, tid);
  fenceProxyAsync();
  __syncthreads();
  refreshThresholds<Metric, Weight, kKnn>(p, m, w, sh, lists, firstRow);

  unsigned long long computed = 0;
  bool failed = false;
  uint32_t mmaPhase = 0;
  const uint32_t idesc = umma_idesc_tf32(128, 128);
  const bool maskPass = useComp && !p.singletons;

  // One staged column tile: operand, MMA, screened epilogue.
  auto processTile = [&](int J, const float *raw, const ColumnMeta &cm, bool colPure) {
    if (tid >= kTile)
      buildColumnOperand(raw, centre, p.d, kPad, scale, opB, sbo, tid - kTile);
    fenceProxyAsync();
    __syncthreads();
    if (tid == 0) {
      tcgenFenceAfter();
      for (int s = 0; s < kPad / 8; ++s)
        mmaTf32(tmem, umma_smem_desc((const char *)opA + 256 * s, 128, sbo),
                umma_smem_desc((const char *)opB + 256 * s, 128, sbo), idesc, s > 0);
      mmaCommit(&mmaBar);
    }
    const bool done = mbarrierWait(&mmaBar, mmaPhase);
    mmaPhase ^= 1;
    if (__syncthreads_or(!done)) {
      failed = true;
      return;
    }
    tcgenFenceAfter();
    if (tid < kTile) {
      const bool mask = maskPass && !(rowPure >= 0 && colPure);
      const uint32_t lane = tmem + ((uint32_t)(warp * 32) << 16);
      float F = sh.rowFilter[myRow];
      float mn = INFINITY;
      float v[32];
#pragma unroll
      for (int chunk = 0; chunk < 4; ++chunk) {
        tmemLoad32(lane + chunk * 32, v);
        if (mask) {
#pragma unroll
          for (int c = 0; c < 32; ++c)
            mn = fminf(mn, cm.comp[chunk * 32 + c] != myComp ? v[c] : INFINITY);
        } else {
#pragma unroll
          for (int c = 0; c < 32; ++c)
            mn = fminf(mn, v[c]);
        }
      }
      if (__any_sync(0xffffffffu, myValid && mn <= F)) {
        unsigned long long best = kEmptyKey;
#pragma unroll 1
        for (int chunk = 0; chunk < 4; ++chunk) {
          tmemLoad32(lane + chunk * 32, v);
          if (!(myValid && mn <= F))
            continue;
          unsigned candidates = 0;
#pragma unroll
          for (int c = 0; c < 32; ++c)
            candidates |= (v[c] <= F ? 1u : 0u) << c;
          while (candidates) {
            const int c = __ffs(candidates) - 1;
            candidates &= candidates - 1;
            const int j = chunk * 32 + c;
            if (J * kTile + j >= p.n)
              continue;
            const int colComp = useComp ? cm.comp[j] : cm.orig[j];
            if (!kKnn && colComp == myComp)
              continue;
            // The reference's exact FP32 distance of the pair.
            typename Metric::Acc acc = m.init();
            for (int k = 0; k < p.d; ++k)
              acc = m.accumulate(acc, sA[k * kTile + myRow], raw[k * kTile + j]);
            if (kKnn) {
              const float value =
                  J * kTile + j == myPos ? 0.0f : fmaxf(m.finalize(acc), 0.0f);
              float *list = lists + myRow * p.k;
              insertSorted(list, p.k, value);
              F = m.filterBound(list[p.k - 1]);
            } else {
              const float weight = w.weight(m.finalize(acc), myVal, useValue ? cm.value[j] : 0.0f);
              if (weight < INFINITY) {
                const unsigned long long key = packKey(weight, (uint32_t)cm.orig[j]);
                best = key < best ? key : best;
              }
            }
          }
        }
        if (!kKnn && best < sh.rowBest[myRow])
          sh.rowBest[myRow] = best;
      }
    }
    tcgenFenceBefore();
    __syncthreads();
    refreshThresholds<Metric, Weight, kKnn>(p, m, w, sh, lists, firstRow);
    ++computed;
  };

  if (rowPure < 0)
    processTile(I, sA, meta[0], false);

  const uint32_t metaBytes = (uint32_t)(kTile * sizeof(int)) * (1 + useComp + useValue);
  const uint32_t tileBytes = (uint32_t)(KC * kTile * sizeof(float));
  auto issue = [&](int i, int b) {
    const int J = sh.listTile[i] & ~kPureColumnTile;
    fenceProxyAsync();
    mbarrierArriveExpectTx(&sh.bar[b], tileBytes + metaBytes);
    bulkCopyToShared(sB[b], p.tiled + (size_t)J * tileFloats, tileBytes, &sh.bar[b]);
    bulkCopyToShared(meta[b].orig, p.order + (size_t)J * kTile, kTile * sizeof(int), &sh.bar[b]);
    if (useComp)
      bulkCopyToShared(meta[b].comp, p.component + (size_t)J * kTile, kTile * sizeof(int),
                       &sh.bar[b]);
    if (useValue)
      bulkCopyToShared(meta[b].value, w.value + (size_t)J * kTile, kTile * sizeof(float),
                       &sh.bar[b]);
  };
  uint32_t phase[2] = {0, 0};
  bool inFlight[2] = {false, false};

  while (!failed) {
    if (tid < 32)
      collectCandidates(p, m, w, sh, rowLow, rowHigh, I, rowPure, rowMinValue, slack);
    __syncthreads();
    const int len = sh.listLen;
    if (sh.overflow) {
      failed = true;
      break;
    }
    if (len == 0 && sh.frontLen == 0)
      break;
    if (p.prune && len > 1)
      sortCandidates(sh, len);
    auto nextValid = [&](int from) {
      while (from < len && sh.listLb[from] > sh.thrTile)
        ++from;
      return from;
    };
    int cur = nextValid(0), buf = 0;
    if (cur < len) {
      if (tid == 0)
        issue(cur, buf);
      inFlight[buf] = true;
    }
    while (cur < len && !failed) {
      const int next = nextValid(cur + 1);
      if (next < len) {
        if (tid == 0)
          issue(next, buf ^ 1);
        inFlight[buf ^ 1] = true;
      }
      const bool ready = mbarrierWait(&sh.bar[buf], phase[buf]);
      phase[buf] ^= 1;
      inFlight[buf] = false;
      if (__syncthreads_or(!ready)) {
        failed = true;
        break;
      }
      if (sh.listLb[cur] <= sh.thrTile)
        processTile(sh.listTile[cur] & ~kPureColumnTile, sB[buf], meta[buf],
                    (sh.listTile[cur] & kPureColumnTile) != 0);
      else
        __syncthreads();
      cur = next;
      buf ^= 1;
    }
    __syncthreads();
    if (sh.frontLen == 0)
      break;
  }

  for (int b = 0; b < 2; ++b)
    if (inFlight[b])
      mbarrierWait(&sh.bar[b], phase[b]);
  if (tid < kTile) {
    const int pos = firstRow + tid;
    if (pos < p.n) {
      if (kKnn)
        p.core[pos] = lists[tid * p.k + p.k - 1];
      else
        p.nearest[pos] = sh.rowBest[tid];
    }
  }
  // Tensor memory goes back before the block leaves, on every path.
  tcgenFenceBefore();
  __syncthreads();
  if (warp == 0) {
    tcgenFenceAfter();
    tmemDealloc(tmem, kTile);
  }
  if (tid == 0) {
    if (p.tilesComputed)
      atomicAdd(p.tilesComputed, computed);
    if (failed && p.error)
      atomicCAS(p.error, 0, sh.overflow ? (int)kErrorTooLarge : (int)kErrorTimeout);
  }
}

// Screen mode set by cuhc_set_screen (0 auto, 1 always where supported,
// 2 never). Results are identical in every mode.
int currentScreenMode();

template <class Metric> struct ScreenSupport {
  static constexpr bool value = false;
};
template <> struct ScreenSupport<EuclideanMetric> {
  static constexpr bool value = true;
};
template <> struct ScreenSupport<SqEuclideanMetric> {
  static constexpr bool value = true;
};

// Dynamic shared memory of a screened pass block (k = 0: nearest pass).
inline size_t screenDynamicBytes(int d, int k) {
  const int kc = chunkWidthFor(d);
  return (size_t)3 * kc * kTile * sizeof(float) + 6 * kTile * sizeof(int) +
         (size_t)2 * kTile * screenK(d) * sizeof(float) + (size_t)(3 * d + kTile * k) * sizeof(float);
}

// Shared memory a block may use on sm_100 (227 KiB).
constexpr size_t kMaxBlockShared = 227 * 1024;

// Whether a pass over d features (k-NN rank k, 0 for a nearest pass) runs
// screened: the metric has a screened form, the features fit one chunk of at
// most 32, the block's shared memory fits, and screening is not switched off.
template <class Metric> inline bool useScreen(int d, int k) {
  return ScreenSupport<Metric>::value && currentScreenMode() != 2 &&
         chunkWidthFor(d) * numChunksFor(d) <= 32 &&
         screenDynamicBytes(d, k) + sizeof(PassState) + 64 <= kMaxBlockShared;
}

// Launches the screened pass; returns a negative code when the metric or the
// dimension has no screened form (callers then use launchPass).
template <class Metric, class Weight, bool kKnn>
int launchScreen(const PassParams &p, const Metric &m, const Weight &w, int kc,
                 cudaStream_t stream) {
  if constexpr (!ScreenSupport<Metric>::value) {
    return kErrorInvalidAlgorithm;
  } else {
    if (p.numChunks != 1)
      return kErrorInvalidAlgorithm;
    const int kPad = screenK(p.d);
    const float margin = screenMargin(p.d);
    if (kc != chunkWidthFor(p.d))
      return kErrorInvalidAlgorithm;
    const size_t dynBytes = screenDynamicBytes(p.d, kKnn ? p.k : 0);
    auto misaligned = [](const void *ptr) { return ((uintptr_t)ptr & 15) != 0; };
    if (misaligned(p.tiled) || misaligned(p.order) || misaligned(p.component) ||
        misaligned(w.value))
      return (int)cudaErrorMisalignedAddress;
    auto run = [&](auto kernel) {
      const cudaError_t e =
          cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dynBytes);
      if (e != cudaSuccess)
        return (int)e;
      kernel<<<p.numTiles, kThreads, dynBytes, stream>>>(p, m, w, margin, kPad);
      noteLaunch();
      return (int)cudaGetLastError();
    };
    switch (kc) {
    case 4:
      return run(screenKernel<Metric, Weight, 4, kKnn>);
    case 8:
      return run(screenKernel<Metric, Weight, 8, kKnn>);
    case 16:
      return run(screenKernel<Metric, Weight, 16, kKnn>);
    default:
      return run(screenKernel<Metric, Weight, 32, kKnn>);
    }
  }
}

} // namespace cuhc
