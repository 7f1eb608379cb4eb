// Core distances by radix select (any k): the route of the reference's
// coreDistancesRadixSelect (hdbscan.cuh:40-105, 293-319) on this engine.
//
// Rows are taken in chunks of whole row tiles whose rows x n distance block
// fits kRadixChunkBytes. The engine's pairwise kernel writes the block (the
// same FP32 arithmetic as every pass, so the same bits); one block of
// kRadixThreads per row then finds the k-th smallest value (the point itself
// counts as distance 0; values are clamped at 0, as in the list path) with
// four 8-bit histogram passes over the float bits, which order like the
// values for non-negative floats. Result: exactly the value the per-row
// k-NN lists produce, for every k <= n. HBM-bound: per chunk the block is
// written once and read four times.
#pragma once

#include <algorithm>

#include "pairwise.cuh"

namespace cuhc {

constexpr size_t kRadixChunkBytes = size_t(512) << 20;
constexpr int kRadixThreads = 512;

// One block per row of the chunk: core[firstRow + row] = k-th smallest of
// dist[row][0..n) with dist[row][firstRow + row] taken as 0.
static __global__ void __launch_bounds__(kRadixThreads)
    radixSelectRowsKernel(const float *__restrict__ dist, int n, int rows, int firstRow, int k,
                          float *__restrict__ core) {
  __shared__ unsigned int hist[256];
  __shared__ unsigned int nextPrefix, nextRemaining;
  const int row = blockIdx.x;
  if (row >= rows)
    return;
  const float *d = dist + (size_t)row * n;
  const int self = firstRow + row;
  const int tid = threadIdx.x, lane = tid & 31;
  unsigned int prefix = 0, remaining = (unsigned int)k;
  for (int pass = 0; pass < 4; ++pass) {
    const int shift = 24 - 8 * pass;
    for (int b = tid; b < 256; b += kRadixThreads)
      hist[b] = 0;
    __syncthreads();
    for (int base = 0; base < n; base += kRadixThreads) {
      const int c = base + tid;
      unsigned int bin = 0xffffffffu;
      if (c < n) {
        const float v = c == self ? 0.0f : fmaxf(d[c], 0.0f);
        const unsigned int key = __float_as_uint(v);
        if (pass == 0 || (key >> (shift + 8)) == prefix)
          bin = (key >> shift) & 255u;
      }
      // One shared-memory add per distinct bin of the warp.
      const unsigned int peers = __match_any_sync(0xffffffffu, bin);
      if (bin != 0xffffffffu && __ffs(peers) - 1 == lane)
        atomicAdd(&hist[bin], (unsigned int)__popc(peers));
    }
    __syncthreads();
    if (tid == 0) {
      unsigned int below = 0;
      for (int b = 0; b < 256; ++b) {
        if (below + hist[b] >= remaining) {
          nextPrefix = (prefix << 8) | (unsigned int)b;
          nextRemaining = remaining - below;
          break;
        }
        below += hist[b];
      }
    }
    __syncthreads();
    prefix = nextPrefix;
    remaining = nextRemaining;
    __syncthreads();
  }
  if (tid == 0)
    core[self] = __uint_as_float(prefix);
}

// core[position] for every position of the index (k-d order), 1 <= k <= n.
template <class Metric>
int coreDistancesRadix(SpatialIndex &index, const Metric &m, int k, float *core,
                       cudaStream_t stream) {
  StatusChain st;
  const int n = index.n;
  const long long rowsFit = (long long)(kRadixChunkBytes / ((size_t)n * sizeof(float)));
  const int chunkTiles = (int)std::max<long long>(1, std::min<long long>(rowsFit / kTile,
                                                                         index.numTiles));
  DeviceBuffer<float> block;
  CUHC_TRY(st, block.allocate((size_t)chunkTiles * kTile * n, stream));
  const size_t tileFloats = index.tileFloats();
  for (int tile0 = 0; tile0 < index.numTiles && st.ok(); tile0 += chunkTiles) {
    const int firstRow = tile0 * kTile;
    const int rows = std::min(chunkTiles * kTile, n - firstRow);
    CUHC_TRY(st, launchPairwise(index.tiled.get() + (size_t)tile0 * tileFloats, index.tiled.get(),
                                rows, n, index.d, m, block.get(), stream));
    radixSelectRowsKernel<<<rows, kRadixThreads, 0, stream>>>(block.get(), n, rows, firstRow, k,
                                                              core);
    noteLaunch();
    CUHC_TRY(st, cudaGetLastError());
  }
  return st.code;
}

} // namespace cuhc
