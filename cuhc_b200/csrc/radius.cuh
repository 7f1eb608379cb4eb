// Learned radius proposal for single-linkage Borůvka rounds (d = 16).
//
// Before a round's nearest pass every point gets 19 features: its 16
// coordinates scaled to [-1, 1] over the data's bounding box, the log of its
// component's size, the round index, and the log of the weight its row found
// in the previous round (0 in round 0). The MLP of mlp.cu predicts the log of
// the row's nearest other-component weight; the proposed radius is
// exp(prediction + offset), offset a calibration margin stored with the
// model. The pass runs with every row's threshold capped by its radius.
// Borůvka needs each component's lightest edge, not each row's, so rows are
// certified per component: with m_C the lightest edge weight any row of
// component C found, a row is done when its best edge weighs at most its
// radius (any lighter pair would lie inside the radius and would have been
// found) or when its radius is at least m_C (every pair of the row up to
// m_C, ties included, was searched, and nothing heavier can be C's lightest
// edge). m_C may also be lowered by any other real edge of C known (the
// component best of the round: last round's edges that leave C). Only the
// other rows -- a radius below m_C and nothing found inside it -- search
// again, in a fallback pass with no cap, whose component bests start at m_C,
// while certified rows sit out. Results never depend on the model; a poor one
// only costs time.
#pragma once

#include <vector>

#include "common.cuh"
#include "spatial.cuh"

namespace cuhc {

constexpr int kRadiusFeatures = 19;
constexpr int kRadiusDims = 16;
constexpr int kRadiusParams = 5505;

int mlpForward(const float *params, const float *x, int count, float *out, cudaStream_t s);

// The model in use (device parameters of the current device), or null.
struct RadiusModel {
  const float *params = nullptr;
  float offset = 0.0f;
};
RadiusModel currentRadiusModel();
// Counters: rows proposed, rows certified by the first pass.
void addRadiusStats(unsigned long long proposed, unsigned long long certified,
                    unsigned long long cappedTiles, unsigned long long fallbackTiles);

// Logging of (features, target) rows for training, filled by a Borůvka run.
struct RadiusLog {
  int maxRowsPerRound = 0;
  unsigned long long seed = 0;
  std::vector<float> features, targets; // [rows][19], [rows]
};

namespace radius_detail {

static __global__ void componentSizes(const int *__restrict__ comp, const int *__restrict__ order,
                                      int n, int *__restrict__ size) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && order[i] >= 0)
    atomicAdd(&size[comp[i]], 1);
}

// features[pos][19] of every position (padding rows get zeros).
static __global__ void radiusFeatures(const float *__restrict__ tiled, int n, int d, int kc,
                                      size_t tileFloats, const int *__restrict__ order,
                                      const float *__restrict__ low,
                                      const float *__restrict__ high,
                                      const int *__restrict__ comp, const int *__restrict__ size,
                                      const unsigned long long *__restrict__ previous, int round,
                                      float *__restrict__ features) {
  const int pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= n)
    return;
  float *f = features + (size_t)pos * kRadiusFeatures;
  if (order[pos] < 0) {
    for (int k = 0; k < kRadiusFeatures; ++k)
      f[k] = 0.0f;
    return;
  }
  const float *tile = tiled + (size_t)(pos / kTile) * tileFloats;
  for (int k = 0; k < d; ++k) {
    const float x = tile[(size_t)((k / kc) * kc + k % kc) * kTile + pos % kTile];
    const float span = high[k] - low[k];
    f[k] = span > 0.0f ? 2.0f * (x - low[k]) / span - 1.0f : 0.0f;
  }
  f[d] = logf((float)size[comp[pos]]);
  f[d + 1] = (float)round;
  const unsigned long long key = previous[pos];
  f[d + 2] = (round > 0 && key != kEmptyKey) ? logf(keyWeight(key) + 1e-30f) : 0.0f;
}

// radius[pos] = exp(prediction + offset) for points, -1 (settled) for padding.
static __global__ void radiusFromPrediction(const float *__restrict__ prediction,
                                            const int *__restrict__ order, int n, float offset,
                                            float *__restrict__ radius) {
  const int pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos < n)
    radius[pos] = order[pos] < 0 ? -1.0f : expf(prediction[pos] + offset);
}

// Tile accounting of the proposal's passes: acc = [mark, capped, fallback];
// step 0 marks the pass counter, step 1 adds the tiles since the mark to the
// capped tiles (and marks again), step 2 to the fallback tiles.
static __global__ void radiusTileStep(const unsigned long long *__restrict__ tiles, int step,
                                      unsigned long long *__restrict__ acc) {
  const unsigned long long now = *tiles;
  if (step > 0)
    acc[step] += now - acc[0];
  acc[0] = now;
}

// After the capped pass: lowers compMin[comp] (float bits of real edge
// weights) to the lightest edge any row of the component found.
static __global__ void componentMinFound(const unsigned long long *__restrict__ nearest,
                                         const int *__restrict__ order,
                                         const int *__restrict__ comp, int n,
                                         unsigned int *__restrict__ compMin) {
  const int pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= n || order[pos] < 0)
    return;
  const unsigned long long key = nearest[pos];
  if (key != kEmptyKey)
    atomicMin(&compMin[comp[pos]], (unsigned int)(key >> 32));
}

// Certification by component (see the header): certified rows get -1
// (settled, their capped result stands), the others +inf (searched again,
// uncapped); counts the certified rows.
static __global__ void certifyRows(const unsigned long long *__restrict__ nearest,
                                   const int *__restrict__ order, const int *__restrict__ comp,
                                   const unsigned int *__restrict__ compMin, int n,
                                   float *__restrict__ radius,
                                   unsigned long long *__restrict__ certified) {
  const int pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= n || order[pos] < 0)
    return;
  const unsigned long long key = nearest[pos];
  const float r = radius[pos];
  const bool inside = key != kEmptyKey && keyWeight(key) <= r;
  const bool ok = inside || r >= __uint_as_float(compMin[comp[pos]]);
  radius[pos] = ok ? -1.0f : INFINITY;
  if (ok)
    atomicAdd(certified, 1ull);
}

// Training target: log of the row's exact nearest other-component weight.
static __global__ void radiusTargets(const unsigned long long *__restrict__ nearest,
                                     const int *__restrict__ order, int n,
                                     float *__restrict__ target) {
  const int pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= n)
    return;
  const unsigned long long key = nearest[pos];
  target[pos] = (order[pos] < 0 || key == kEmptyKey) ? NAN : logf(keyWeight(key) + 1e-30f);
}

} // namespace radius_detail
} // namespace cuhc
