// Ward by the nearest-neighbour chain, in one persistent cooperative kernel.
//
// The chain algorithm (reducible linkage): look up the nearest active
// cluster of the chain's top; if it is the cluster below the top, merge the
// two, else push it. Same rules and formulas as the reference's chain
// (nn_chain.cuh:46-289): the cluster below the top wins ties, other ties go
// to the lower slot, merged centroid c_top + (c_b - c_top) n_b / (n_top + n_b)
// in the lower slot, height sqrt(2 n_a n_b / (n_a + n_b) |c_a - c_b|^2).
//
// Each step every block scans its slot range, then block 0 combines and
// updates the chain. The two grid-wide barriers per step are this library's
// own: an arrival counter and a generation word, every wait bounded by an
// iteration limit. A wait that runs out records kErrorTimeout and the block
// returns; the host reports the error. The launch is cooperative, so all
// blocks are co-resident.
#include "asyncload.cuh"
#include "profiling.cuh"
#include "rnn.cuh"

#include <vector>

namespace cuhc {
namespace {

constexpr int kChainThreads = 256;

struct ChainState {
  float *cent;        // m x d, slot order
  int *size;          // 0 = retired
  int *chain, *chainLength, *current, *nextStart;
  float *blockDist;   // per block best
  int *blockSlot;
  int *mergeA, *mergeB;
  float *mergeH;
  int *numMerges;
  unsigned int *barrierCount, *barrierGen;
  int *error;
  int m, d;
};

__device__ __forceinline__ bool lessLoc(float da, int ia, float db, int ib) {
  return da < db || (da == db && ia < ib);
}

// Grid barrier with a bounded wait. Returns false (everyone in the block)
// when the wait ran out (after spinLimit polls; only the bounded-wait
// self-test passes a shorter limit).
__device__ bool gridBarrier(const ChainState &s, long long spinLimit = kSpinLimit) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    volatile unsigned int *gen = s.barrierGen;
    const unsigned int g = *gen;
    __threadfence();
    if (atomicAdd(s.barrierCount, 1u) == gridDim.x - 1) {
      *s.barrierCount = 0;
      __threadfence();
      atomicAdd(s.barrierGen, 1u);
    } else {
      long long spins = 0;
      while (*gen == g) {
        if (++spins > spinLimit) {
          atomicCAS(s.error, 0, (int)kErrorTimeout);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
  }
  __syncthreads();
  return ok != 0;
}

// b is read through L2 (__ldcg): block 0 rewrites merged centroids, and the
// other blocks' L1 would otherwise keep stale lines across steps.
__device__ __forceinline__ float wardSquared(const float *a, const float *b, int d, float sa,
                                             float sb) {
  float squared = 0.0f;
  for (int k = 0; k < d; ++k) {
    const float diff = a[k] - __ldcg(b + k);
    squared = fmaf(diff, diff, squared);
  }
  return 2.0f * sa * sb / (sa + sb) * squared;
}

// Bounded-wait self-test (cuhc_wait_selftest). The grid barrier above with
// block `missing` returning before it arrives: every other block's wait runs
// out after spinLimit polls and records kErrorTimeout. missing < 0: all
// arrive and the barrier completes.
__global__ void barrierSelftestKernel(ChainState s, int missing, long long spinLimit) {
  if ((int)blockIdx.x == missing)
    return;
  gridBarrier(s, spinLimit);
}

// The pass kernels' mbarrier wait on a barrier whose expected arrival never
// comes (missing != 0: nothing arrives) or has come (missing == 0): a wait
// that runs out records kErrorTimeout.
__global__ void mbarrierSelftestKernel(int missing, unsigned long long limitNs, int *error) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbarrierInit(&bar, 1);
    fenceBarrierInit();
  }
  __syncthreads();
  if (threadIdx.x == 0 && !missing)
    mbarrierArrive(&bar, 1);
  if (!mbarrierWait(&bar, 0, limitNs))
    atomicCAS(error, 0, (int)kErrorTimeout);
}

__global__ void __launch_bounds__(kChainThreads) chainKernel(ChainState s) {
  extern __shared__ float topCent[]; // d floats: the chain top's centroid
  __shared__ int top, below, mergeWith;
  __shared__ float redDist[kChainThreads / 32];
  __shared__ int redSlot[kChainThreads / 32];
  const int perBlock = (s.m + gridDim.x - 1) / gridDim.x;
  const int first = blockIdx.x * perBlock, last = min(s.m, first + perBlock);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;

  while (true) {
    if (threadIdx.x == 0) {
      top = __ldcg(s.current);
      const int len = __ldcg(s.chainLength);
      below = len >= 2 ? __ldcg(s.chain + len - 2) : -1;
    }
    __syncthreads();
    const int a = top, prev = below;
    if (a < 0)
      return;
    for (int k = threadIdx.x; k < s.d; k += kChainThreads)
      topCent[k] = __ldcg(s.cent + (size_t)a * s.d + k);
    __syncthreads();
    const float sa = (float)__ldcg(s.size + a);
    float best = INFINITY;
    int bestSlot = 0x7fffffff;
    for (int slot = first + threadIdx.x; slot < last; slot += kChainThreads) {
      const int sz = __ldcg(s.size + slot);
      if (sz == 0 || slot == a)
        continue;
      const float dist =
          wardSquared(topCent, (const float *)s.cent + (size_t)slot * s.d, s.d, sa, (float)sz);
      const int idx = slot == prev ? -1 : slot;
      if (lessLoc(dist, idx, best, bestSlot)) {
        best = dist;
        bestSlot = idx;
      }
    }
    for (int off = 16; off > 0; off /= 2) {
      const float od = __shfl_xor_sync(0xffffffffu, best, off);
      const int os = __shfl_xor_sync(0xffffffffu, bestSlot, off);
      if (lessLoc(od, os, best, bestSlot)) {
        best = od;
        bestSlot = os;
      }
    }
    if (lane == 0) {
      redDist[warp] = best;
      redSlot[warp] = bestSlot;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < kChainThreads / 32; ++w)
        if (lessLoc(redDist[w], redSlot[w], best, bestSlot)) {
          best = redDist[w];
          bestSlot = redSlot[w];
        }
      s.blockDist[blockIdx.x] = best;
      s.blockSlot[blockIdx.x] = bestSlot;
    }
    if (!gridBarrier(s))
      return;

    if (blockIdx.x == 0) {
      if (threadIdx.x == 0) {
        float d0 = INFINITY;
        int s0 = 0x7fffffff;
        for (int b = 0; b < (int)gridDim.x; ++b) {
          const float db = __ldcg(s.blockDist + b);
          const int sb = __ldcg(s.blockSlot + b);
          if (lessLoc(db, sb, d0, s0)) {
            d0 = db;
            s0 = sb;
          }
        }
        const int nearest = s0 == -1 ? prev : s0;
        redDist[0] = d0;
        if (nearest < 0 || nearest >= s.m) {
          // No comparable candidate (NaN distances): stop with an error.
          atomicCAS(s.error, 0, (int)kErrorNonFinite);
          mergeWith = -1;
          *s.current = -1;
        } else if (nearest == prev) {
          mergeWith = prev;
        } else {
          mergeWith = -1;
          s.chain[(*s.chainLength)++] = nearest;
          *s.current = nearest;
        }
      }
      __syncthreads();
      if (mergeWith >= 0) {
        const int b = mergeWith;
        const int keep = min(a, b), retire = max(a, b);
        const float sb = (float)__ldcg(s.size + b);
        const float weightB = sb / (sa + sb);
        for (int k = threadIdx.x; k < s.d; k += kChainThreads)
          s.cent[(size_t)keep * s.d + k] =
              fmaf(__ldcg(s.cent + (size_t)b * s.d + k) - topCent[k], weightB, topCent[k]);
        if (threadIdx.x == 0) {
          const int idx = (*s.numMerges)++;
          s.mergeA[idx] = keep;
          s.mergeB[idx] = retire;
          s.mergeH[idx] = sqrtf(redDist[0]);
          s.size[keep] = s.size[a] + s.size[b];
          s.size[retire] = 0;
          *s.chainLength -= 2;
          if (*s.numMerges == s.m - 1) {
            *s.current = -1;
          } else if (*s.chainLength > 0) {
            *s.current = s.chain[*s.chainLength - 1];
          } else {
            int start = *s.nextStart;
            while (start < s.m && s.size[start] == 0)
              ++start;
            *s.nextStart = start;
            s.chain[0] = start;
            *s.chainLength = 1;
            *s.current = start < s.m ? start : -1;
          }
        }
      }
      __threadfence();
    }
    if (!gridBarrier(s))
      return;
  }
}

} // namespace

int chainOnClusters(const float *centroids, const int *sizes, int m, int d, cudaStream_t stream,
                    std::vector<int> &a, std::vector<int> &b, std::vector<float> &h) {
  a.clear();
  b.clear();
  h.clear();
  if (m < 2)
    return 0;
  int device = 0, coop = 0, sms = 0, perSm = 0;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
  if (!coop)
    return (int)cudaErrorNotSupported;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const size_t shared = (size_t)d * sizeof(float);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, chainKernel, kChainThreads, shared);
  const int numBlocks = std::max(1, std::min(perSm * sms, (m + kChainThreads - 1) / kChainThreads));
  StatusChain st;
  DeviceBuffer<float> cent, blockDist, mergeH;
  DeviceBuffer<int> size, chain, scalars, blockSlot, mergeA, mergeB;
  DeviceBuffer<unsigned int> barrier;
  CUHC_TRY(st, cent.allocate((size_t)m * d, stream));
  CUHC_TRY(st, size.allocate(m, stream));
  CUHC_TRY(st, chain.allocate(m, stream));
  CUHC_TRY(st, scalars.allocate(5, stream)); // chainLength, current, nextStart, numMerges, error
  CUHC_TRY(st, blockDist.allocate(numBlocks, stream));
  CUHC_TRY(st, blockSlot.allocate(numBlocks, stream));
  CUHC_TRY(st, mergeA.allocate(m - 1, stream));
  CUHC_TRY(st, mergeB.allocate(m - 1, stream));
  CUHC_TRY(st, mergeH.allocate(m - 1, stream));
  CUHC_TRY(st, barrier.allocate(2, stream));
  if (!st.ok())
    return st.code;
  CUHC_TRY(st, cudaMemcpyAsync(cent.get(), centroids, cent.bytes(), cudaMemcpyDeviceToDevice,
                               stream));
  CUHC_TRY(st, cudaMemcpyAsync(size.get(), sizes, size.bytes(), cudaMemcpyDeviceToDevice, stream));
  const int init[5] = {1, 0, 0, 0, 0};
  CUHC_TRY(st, cudaMemcpyAsync(scalars.get(), init, sizeof(init), cudaMemcpyHostToDevice, stream));
  CUHC_TRY(st, cudaMemsetAsync(chain.get(), 0, sizeof(int), stream));
  CUHC_TRY(st, cudaMemsetAsync(barrier.get(), 0, 2 * sizeof(unsigned int), stream));
  ChainState s{};
  s.cent = cent.get();
  s.size = size.get();
  s.chain = chain.get();
  s.chainLength = scalars.get();
  s.current = scalars.get() + 1;
  s.nextStart = scalars.get() + 2;
  s.numMerges = scalars.get() + 3;
  s.error = scalars.get() + 4;
  s.blockDist = blockDist.get();
  s.blockSlot = blockSlot.get();
  s.mergeA = mergeA.get();
  s.mergeB = mergeB.get();
  s.mergeH = mergeH.get();
  s.barrierCount = barrier.get();
  s.barrierGen = barrier.get() + 1;
  s.m = m;
  s.d = d;
  void *args[] = {&s};
  CUHC_TRY(st, cudaLaunchCooperativeKernel((void *)chainKernel, numBlocks, kChainThreads, args,
                                           shared, stream));
  noteLaunch();
  int hostScalars[5] = {};
  CUHC_TRY(st, cudaMemcpyAsync(hostScalars, scalars.get(), sizeof(hostScalars),
                               cudaMemcpyDeviceToHost, stream));
  CUHC_TRY(st, cudaStreamSynchronize(stream));
  if (st.ok() && hostScalars[4])
    st(hostScalars[4]);
  if (st.ok() && hostScalars[3] != m - 1)
    st(kErrorNonFinite);
  if (!st.ok())
    return st.code;
  a.resize(m - 1);
  b.resize(m - 1);
  h.resize(m - 1);
  CUHC_TRY(st, cudaMemcpyAsync(a.data(), mergeA.get(), (m - 1) * sizeof(int),
                               cudaMemcpyDeviceToHost, stream));
  CUHC_TRY(st, cudaMemcpyAsync(b.data(), mergeB.get(), (m - 1) * sizeof(int),
                               cudaMemcpyDeviceToHost, stream));
  CUHC_TRY(st, cudaMemcpyAsync(h.data(), mergeH.get(), (m - 1) * sizeof(float),
                               cudaMemcpyDeviceToHost, stream));
  CUHC_TRY(st, cudaStreamSynchronize(stream));
  return st.code;
}

} // namespace cuhc

// Self-test of the bounded device waits: a wait whose arrival never comes
// must run out and report kErrorTimeout, leaving the context usable; with
// every arrival made it must complete. No fault, trap or unbounded spin is
// involved: the missing arrival is a block that returns early (grid barrier)
// or an arrival that is never made (mbarrier).
extern "C" int cuhc_wait_selftest(int kind, int missing, int limitMicroseconds) {
  using namespace cuhc;
  if (kind < 0 || kind > 1 || limitMicroseconds < 1 || limitMicroseconds > 1000000)
    return kErrorInvalidShape;
  cudaStream_t stream = nullptr;
  StatusChain st;
  st((int)cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  DeviceBuffer<unsigned int> words;
  CUHC_TRY(st, words.allocate(3, stream)); // barrier count, generation, error
  CUHC_TRY(st, cudaMemsetAsync(words.get(), 0, words.bytes(), stream));
  int *error = reinterpret_cast<int *>(words.get() + 2);
  if (st.ok() && kind == 0) {
    ChainState s{};
    s.barrierCount = words.get();
    s.barrierGen = words.get() + 1;
    s.error = error;
    int absent = missing ? 1 : -1;
    // A poll takes at least the 64 ns nap: about 8 polls per microsecond.
    long long polls = 8ll * limitMicroseconds;
    void *args[] = {&s, &absent, &polls};
    CUHC_TRY(st, cudaLaunchCooperativeKernel((void *)barrierSelftestKernel, 4, 32, args, 0,
                                             stream));
    noteLaunch();
  } else if (st.ok()) {
    mbarrierSelftestKernel<<<1, 32, 0, stream>>>(missing, 1000ull * limitMicroseconds, error);
    noteLaunch();
    CUHC_TRY(st, cudaGetLastError());
  }
  int recorded = 0;
  CUHC_TRY(st, cudaMemcpyAsync(&recorded, error, sizeof(int), cudaMemcpyDeviceToHost, stream));
  CUHC_TRY(st, cudaStreamSynchronize(stream));
  words.release();
  if (stream) {
    cudaStreamSynchronize(stream);
    cudaStreamDestroy(stream);
  }
  return st.ok() ? recorded : st.code;
}
