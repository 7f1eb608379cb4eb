// Full distance matrix (cuhc_pairwise_distances): the engine's tile loop
// with a store epilogue, one block per 128 x 128 output tile. Same per-pair
// arithmetic as every pass, so the matrix equals the reference's
// pairwiseDistanceKernel (distance_matrix.cuh:177-200) bit for bit.
#pragma once

#include "profiling.cuh"
#include "engine.cuh"

namespace cuhc {

// A tiled copy of points in their original order (no spatial index).
int buildTiled(const float *points, int n, int d, DeviceBuffer<float> &tiled, cudaStream_t s);

template <class Metric, int KC>
__global__ void __launch_bounds__(kThreads, 2)
    pairwiseKernel(const float *__restrict__ tiledA, const float *__restrict__ tiledB, int nA,
                   int nB, int numChunks, Metric m, float *__restrict__ out) {
  extern __shared__ __align__(128) float dyn[];
  float *sA = dyn, *sB = dyn + KC * kTile;
  const TileGeom g;
  const int I = blockIdx.y, J = blockIdx.x;
  if (numChunks == 1)
    copyChunk(sA, tiledA + (size_t)I * KC * kTile, KC * kTile);
  typename Metric::Acc acc[8][8];
  computeTile<Metric, KC>(tiledA, tiledB, numChunks, I, J, sA, sB, m, acc, g);
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const long long row = (long long)I * kTile + g.row(r);
    if (row >= nA)
      continue;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int col = J * kTile + g.col(c);
      if (col < nB)
        out[row * nB + col] = m.finalize(acc[r][c]);
    }
  }
}

template <class Metric>
int launchPairwise(const float *tiledA, const float *tiledB, int nA, int nB, int d,
                   const Metric &m, float *out, cudaStream_t s) {
  const int kc = chunkWidthFor(d), numChunks = numChunksFor(d);
  const dim3 grid(numTilesFor(nB), numTilesFor(nA));
  const size_t dyn = 2 * (size_t)kc * kTile * sizeof(float);
  switch (kc) {
  case 4:
    pairwiseKernel<Metric, 4><<<grid, kThreads, dyn, s>>>(tiledA, tiledB, nA, nB, numChunks, m, out); noteLaunch();
    break;
  case 8:
    pairwiseKernel<Metric, 8><<<grid, kThreads, dyn, s>>>(tiledA, tiledB, nA, nB, numChunks, m, out); noteLaunch();
    break;
  case 16:
    pairwiseKernel<Metric, 16><<<grid, kThreads, dyn, s>>>(tiledA, tiledB, nA, nB, numChunks, m, out); noteLaunch();
    break;
  default:
    pairwiseKernel<Metric, 32><<<grid, kThreads, dyn, s>>>(tiledA, tiledB, nA, nB, numChunks, m, out); noteLaunch();
    break;
  }
  return (int)cudaGetLastError();
}

template <class Metric>
int pairwiseDistances(const float *A, int nA, const float *B, int nB, int d, const Metric &m,
                      float *out, cudaStream_t s);

} // namespace cuhc
