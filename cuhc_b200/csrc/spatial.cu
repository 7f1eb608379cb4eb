// GPU k-d ordering, tiled layout and BVH summaries (see spatial.cuh).
#include "profiling.cuh"
#include "spatial.cuh"

#include <algorithm>
#include <cstring>
#include <vector>
#include <cub/device/device_radix_sort.cuh>

namespace cuhc {

void BvhTopology::build(int T) {
  numTiles = T;
  left.clear();
  right.clear();
  firstTile.clear();
  tileCount.clear();
  levelStart.clear();
  leafOfTile.assign(T, -1);
  if (T <= 0) {
    numNodes = depth = 0;
    return;
  }
  firstTile.push_back(0);
  tileCount.push_back(T);
  left.push_back(-1);
  right.push_back(-1);
  levelStart.push_back(0);
  int begin = 0;
  while (begin < (int)firstTile.size()) {
    const int end = (int)firstTile.size();
    for (int node = begin; node < end; ++node) {
      const int first = firstTile[node], count = tileCount[node];
      if (count == 1) {
        leafOfTile[first] = node;
        continue;
      }
      const int leftCount = count / 2;
      left[node] = (int)firstTile.size();
      firstTile.push_back(first);
      tileCount.push_back(leftCount);
      left.push_back(-1);
      right.push_back(-1);
      right[node] = (int)firstTile.size();
      firstTile.push_back(first + leftCount);
      tileCount.push_back(count - leftCount);
      left.push_back(-1);
      right.push_back(-1);
    }
    begin = end;
    if (begin < (int)firstTile.size())
      levelStart.push_back(begin);
  }
  levelStart.push_back((int)firstTile.size());
  numNodes = (int)firstTile.size();
  depth = (int)levelStart.size() - 1;
  spans.assign(numNodes, 0);
  rootOfInstance.assign(1, 0);
}

void BvhTopology::buildForest(const std::vector<int> &instanceTiles) {
  std::vector<int> start(instanceTiles.size() + 1, 0);
  for (size_t i = 0; i < instanceTiles.size(); ++i)
    start[i + 1] = start[i] + instanceTiles[i];
  const int T = start.back();
  numTiles = T;
  left.clear();
  right.clear();
  firstTile.clear();
  tileCount.clear();
  levelStart.clear();
  spans.clear();
  leafOfTile.assign(T, -1);
  rootOfInstance.assign(instanceTiles.size(), -1);
  // Instance holding a tile: the last start <= tile.
  auto instanceOf = [&](int tile) {
    return (int)(std::upper_bound(start.begin(), start.end(), tile) - start.begin()) - 1;
  };
  auto addNode = [&](int first, int count) {
    firstTile.push_back(first);
    tileCount.push_back(count);
    left.push_back(-1);
    right.push_back(-1);
    spans.push_back(0);
    return (int)firstTile.size() - 1;
  };
  addNode(0, T);
  levelStart.push_back(0);
  int begin = 0;
  while (begin < (int)firstTile.size()) {
    const int end = (int)firstTile.size();
    for (int node = begin; node < end; ++node) {
      const int first = firstTile[node], count = tileCount[node];
      const int a = instanceOf(first), b = instanceOf(first + count - 1);
      if (a == b && rootOfInstance[a] < 0)
        rootOfInstance[a] = node;
      if (count == 1) {
        leafOfTile[first] = node;
        continue;
      }
      int leftCount;
      if (a != b) {
        // The boundary start[a + 1 .. b] nearest the middle tile.
        const int middle = first + count / 2;
        int best = start[a + 1];
        for (int i = a + 1; i <= b; ++i)
          if (std::abs(start[i] - middle) < std::abs(best - middle))
            best = start[i];
        leftCount = best - first;
        spans[node] = 1;
      } else {
        leftCount = count / 2;
      }
      const int l = addNode(first, leftCount);
      const int r = addNode(first + leftCount, count - leftCount);
      left[node] = l;
      right[node] = r;
    }
    begin = end;
    if (begin < (int)firstTile.size())
      levelStart.push_back(begin);
  }
  levelStart.push_back((int)firstTile.size());
  numNodes = (int)firstTile.size();
  depth = (int)levelStart.size() - 1;
}

namespace {

constexpr int kSplitSamples = 256;

// One warp per internal node of a level: the feature with the widest spread
// among up to 256 evenly strided points of the node's range.
__global__ void chooseSplitKernel(const float *__restrict__ points, int n, int d,
                                  const int *__restrict__ order, const int *__restrict__ firstTile,
                                  const int *__restrict__ tileCount, int levelBegin, int levelEnd,
                                  int *__restrict__ splitFeature) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32, lane = threadIdx.x % 32;
  const int node = levelBegin + warp;
  if (node >= levelEnd)
    return;
  if (tileCount[node] <= 1) {
    if (lane == 0)
      splitFeature[node] = 0;
    return;
  }
  const int a = firstTile[node] * kTile;
  const int b = min(n, (firstTile[node] + tileCount[node]) * kTile);
  const int len = b - a;
  const int step = max(1, len / kSplitSamples);
  const int samples = min(kSplitSamples, (len + step - 1) / step);
  float bestSpread = -1.0f;
  int bestFeature = 0;
  for (int f = 0; f < d; ++f) {
    float lo = INFINITY, hi = -INFINITY;
    for (int s = lane; s < samples; s += 32) {
      const int o = order[a + s * step];
      if (o < 0)
        continue; // padding slot of a batch
      const float v = points[(size_t)o * d + f];
      lo = fminf(lo, v);
      hi = fmaxf(hi, v);
    }
    for (int off = 16; off > 0; off /= 2) {
      lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, off));
      hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, off));
    }
    if (hi - lo > bestSpread) {
      bestSpread = hi - lo;
      bestFeature = f;
    }
  }
  if (lane == 0)
    splitFeature[node] = bestFeature;
}

// The node of depth `level` (or the leaf above it) that holds a tile.
__device__ __forceinline__ int nodeAtDepth(int tile, int level, const int *left, const int *right,
                                           const int *firstTile, const int *tileCount) {
  int node = 0;
  for (int l = 0; l < level && tileCount[node] > 1; ++l)
    node = tile < firstTile[right[node]] ? left[node] : right[node];
  return node;
}

// Sort keys of one level: (first tile of the position's node) << 32 | the
// order-preserving bits of the split feature; positions in nodes that are
// already single tiles keep their place.
__global__ void levelKeysKernel(const float *__restrict__ points, int n, int d, int level,
                                const int *__restrict__ order, const int *__restrict__ left,
                                const int *__restrict__ right, const int *__restrict__ firstTile,
                                const int *__restrict__ tileCount,
                                const int *__restrict__ splitFeature,
                                const unsigned char *__restrict__ spans,
                                unsigned long long *__restrict__ keys) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n)
    return;
  const int node = nodeAtDepth(p / kTile, level, left, right, firstTile, tileCount);
  uint32_t low;
  if (tileCount[node] == 1 || (spans && spans[node]))
    low = (uint32_t)p; // single tiles and nodes over several instances keep their order
  else if (order[p] < 0)
    low = 0xffffffffu; // padding stays behind its instance's points
  else
    low = orderedBits(points[(size_t)order[p] * d + splitFeature[node]]);
  keys[p] = ((unsigned long long)firstTile[node] << 32) | low;
}

__global__ void iotaKernel(int *out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    out[i] = i;
}

// tiled[tile][chunk][k][row] = points[order[position]][chunk * kc + k];
// padding stays zero (the buffer is cleared first). Also rank = order^-1.
__global__ void gatherTiledKernel(const float *__restrict__ points, int n, int d, int kc,
                                  int numChunks, const int *__restrict__ order,
                                  float *__restrict__ tiled, int *__restrict__ rank) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n)
    return;
  const int o = order ? order[p] : p;
  if (o < 0)
    return; // padding slot of a batch: stays zero
  if (rank)
    rank[o] = p;
  const int t = p / kTile, r = p % kTile;
  float *tileBase = tiled + (size_t)t * numChunks * kc * kTile;
  const float *row = points + (size_t)o * d;
  for (int f = 0; f < d; ++f)
    tileBase[((size_t)(f / kc) * kc + f % kc) * kTile + r] = row[f];
}

// One warp per tile: per-feature min / max over its valid points.
__global__ void leafBoxKernel(const float *__restrict__ tiled, int n, int d, int kc, int numChunks,
                              int numTiles, const int *__restrict__ leafOfTile,
                              const int *__restrict__ padOrder, float *__restrict__ low,
                              float *__restrict__ high) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32, lane = threadIdx.x % 32;
  if (warp >= numTiles)
    return;
  const int t = warp, node = leafOfTile[t];
  const int valid = min(kTile, n - t * kTile);
  const float *tileBase = tiled + (size_t)t * numChunks * kc * kTile;
  for (int f = 0; f < d; ++f) {
    const float4 v =
        *(const float4 *)(tileBase + ((size_t)(f / kc) * kc + f % kc) * kTile + lane * 4);
    const float vals[4] = {v.x, v.y, v.z, v.w};
    float lo = INFINITY, hi = -INFINITY;
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (lane * 4 + i < valid && (!padOrder || padOrder[t * kTile + lane * 4 + i] >= 0)) {
        lo = fminf(lo, vals[i]);
        hi = fmaxf(hi, vals[i]);
      }
    for (int off = 16; off > 0; off /= 2) {
      lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, off));
      hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, off));
    }
    if (lane == 0) {
      low[(size_t)node * d + f] = lo;
      high[(size_t)node * d + f] = hi;
    }
  }
}

__global__ void internalBoxKernel(int levelBegin, int levelEnd, int d, const int *__restrict__ left,
                                  const int *__restrict__ right, float *__restrict__ low,
                                  float *__restrict__ high) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long total = (long long)(levelEnd - levelBegin) * d;
  if (e >= total)
    return;
  const int node = levelBegin + (int)(e / d), f = (int)(e % d);
  const int l = left[node], r = right[node];
  if (l < 0)
    return;
  low[(size_t)node * d + f] = fminf(low[(size_t)l * d + f], low[(size_t)r * d + f]);
  high[(size_t)node * d + f] = fmaxf(high[(size_t)l * d + f], high[(size_t)r * d + f]);
}

// One warp per tile: smallest value and purity of the leaf.
__global__ void leafSummaryKernel(int n, int numTiles, const int *__restrict__ leafOfTile,
                                  const float *__restrict__ values,
                                  const int *__restrict__ component, float *__restrict__ minValue,
                                  int *__restrict__ pure) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32, lane = threadIdx.x % 32;
  if (warp >= numTiles)
    return;
  const int t = warp, node = leafOfTile[t];
  const int first = t * kTile, valid = min(kTile, n - first);
  float lo = INFINITY;
  int cmin = 0x7fffffff, cmax = -1;
  for (int i = lane; i < valid; i += 32) {
    if (values)
      lo = fminf(lo, values[first + i]);
    if (component) {
      const int c = component[first + i];
      cmin = min(cmin, c);
      cmax = max(cmax, c);
    }
  }
  for (int off = 16; off > 0; off /= 2) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, off));
    cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, off));
    cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, off));
  }
  if (lane == 0) {
    if (minValue)
      minValue[node] = values ? lo : 0.0f;
    if (pure)
      pure[node] = (component && cmin == cmax) ? cmin : -1;
  }
}

__global__ void internalSummaryKernel(int levelBegin, int levelEnd, const int *__restrict__ left,
                                      const int *__restrict__ right, float *__restrict__ minValue,
                                      int *__restrict__ pure) {
  const int node = levelBegin + blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= levelEnd)
    return;
  const int l = left[node], r = right[node];
  if (l < 0)
    return;
  if (minValue)
    minValue[node] = fminf(minValue[l], minValue[r]);
  if (pure)
    pure[node] = (pure[l] >= 0 && pure[l] == pure[r]) ? pure[l] : -1;
}

int blocksFor(long long work, int threads) { return (int)((work + threads - 1) / threads); }

} // namespace

int SpatialIndex::build(const float *points, int n_, int d_, bool spatial, cudaStream_t s) {
  numInstances = 1;
  numPads = 0;
  numPoints = n_;
  instanceFirstTile.assign(1, 0);
  topo.build(numTilesFor(n_));
  return buildCommon(points, n_, d_, spatial, nullptr, s);
}

int SpatialIndex::buildBatch(const float *points, const std::vector<int> &sizes, int d_,
                             cudaStream_t s) {
  numInstances = (int)sizes.size();
  std::vector<int> tiles(sizes.size());
  instanceFirstTile.assign(sizes.size(), 0);
  long long total = 0;
  int tileSum = 0;
  for (size_t i = 0; i < sizes.size(); ++i) {
    tiles[i] = numTilesFor(sizes[i]);
    instanceFirstTile[i] = tileSum;
    tileSum += tiles[i];
    total += sizes[i];
  }
  numPoints = (int)total;
  topo.buildForest(tiles);
  const int positions = tileSum * kTile;
  numPads = positions - numPoints;
  // Instance i's rows start on its first tile; the rest of its last tile is padding.
  std::vector<int> hostOrder(positions, -1);
  long long offset = 0;
  for (size_t i = 0; i < sizes.size(); ++i) {
    const int base = instanceFirstTile[i] * kTile;
    for (int j = 0; j < sizes[i]; ++j)
      hostOrder[base + j] = (int)(offset + j);
    offset += sizes[i];
  }
  return buildCommon(points, positions, d_, true, &hostOrder, s);
}

int SpatialIndex::buildCommon(const float *points, int positions, int d_, bool spatial,
                              const std::vector<int> *hostOrder, cudaStream_t s) {
  n = positions;
  d = d_;
  stream = s;
  numTiles = topo.numTiles;
  kc = chunkWidthFor(d);
  numChunks = numChunksFor(d);
  StatusChain st;
  const int N = topo.numNodes;
  CUHC_TRY(st, order.allocate(paddedToTiles(n), s));
  CUHC_TRY(st, rank.allocate(std::max(numPoints, 1), s));
  CUHC_TRY(st, nodeLeft.allocate(N, s));
  CUHC_TRY(st, nodeRight.allocate(N, s));
  CUHC_TRY(st, nodeFirstTile.allocate(N, s));
  CUHC_TRY(st, nodeTileCount.allocate(N, s));
  CUHC_TRY(st, leafOfTile.allocate(numTiles, s));
  CUHC_TRY(st, nodeLow.allocate((size_t)N * d, s));
  CUHC_TRY(st, nodeHigh.allocate((size_t)N * d, s));
  CUHC_TRY(st, nodeMinValue.allocate(N, s));
  CUHC_TRY(st, nodePure.allocate(N, s));
  CUHC_TRY(st, tiled.allocate((size_t)numTiles * tileFloats(), s));
  if (!st.ok())
    return st.code;
  CUHC_TRY(st, cudaMemcpyAsync(nodeLeft.get(), topo.left.data(), N * sizeof(int),
                               cudaMemcpyHostToDevice, s));
  CUHC_TRY(st, cudaMemcpyAsync(nodeRight.get(), topo.right.data(), N * sizeof(int),
                               cudaMemcpyHostToDevice, s));
  CUHC_TRY(st, cudaMemcpyAsync(nodeFirstTile.get(), topo.firstTile.data(), N * sizeof(int),
                               cudaMemcpyHostToDevice, s));
  CUHC_TRY(st, cudaMemcpyAsync(nodeTileCount.get(), topo.tileCount.data(), N * sizeof(int),
                               cudaMemcpyHostToDevice, s));
  CUHC_TRY(st, cudaMemcpyAsync(leafOfTile.get(), topo.leafOfTile.data(), numTiles * sizeof(int),
                               cudaMemcpyHostToDevice, s));
  if (hostOrder) {
    CUHC_TRY(st, nodeSpans.allocate(N, s));
    CUHC_TRY(st, rootOfTile.allocate(numTiles, s));
    std::vector<int> roots(numTiles);
    for (int i = 0; i < numInstances; ++i) {
      const int last = i + 1 < numInstances ? instanceFirstTile[i + 1] : numTiles;
      for (int t = instanceFirstTile[i]; t < last; ++t)
        roots[t] = topo.rootOfInstance[i];
    }
    CUHC_TRY(st, cudaMemcpyAsync(nodeSpans.get(), topo.spans.data(), N, cudaMemcpyHostToDevice,
                                 s));
    CUHC_TRY(st, cudaMemcpyAsync(rootOfTile.get(), roots.data(), numTiles * sizeof(int),
                                 cudaMemcpyHostToDevice, s));
    CUHC_TRY(st, cudaMemcpyAsync(order.get(), hostOrder->data(), n * sizeof(int),
                                 cudaMemcpyHostToDevice, s));
    // The host vectors go out of scope on return: wait for the copies.
    CUHC_TRY(st, cudaStreamSynchronize(s));
  } else {
    // Positions past the last point are padding (order -1).
    CUHC_TRY(st, cudaMemsetAsync(order.get(), 0xff, paddedToTiles(n) * sizeof(int), s));
    iotaKernel<<<blocksFor(n, 256), 256, 0, s>>>(order.get(), n); noteLaunch();
  }
  CUHC_TRY(st, cudaGetLastError());

  if (spatial && topo.depth > 1 && st.ok()) {
    DeviceBuffer<unsigned long long> keys, keysOut;
    DeviceBuffer<int> valsOut, split;
    CUHC_TRY(st, keys.allocate(n, s));
    CUHC_TRY(st, keysOut.allocate(n, s));
    CUHC_TRY(st, valsOut.allocate(n, s));
    CUHC_TRY(st, split.allocate(N, s));
    int tileBits = 1;
    while ((1 << tileBits) <= numTiles)
      ++tileBits;
    size_t tempBytes = 0;
    CUHC_TRY(st, cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, keys.get(), keysOut.get(),
                                                 order.get(), valsOut.get(), n, 0, 32 + tileBits,
                                                 s));
    DeviceBuffer<unsigned char> temp;
    CUHC_TRY(st, temp.allocate(tempBytes, s));
    // Levels whose nodes still have children.
    for (int level = 0; level + 1 < topo.depth && st.ok(); ++level) {
      const int lb = topo.levelStart[level], le = topo.levelStart[level + 1];
      chooseSplitKernel<<<blocksFor((long long)(le - lb) * 32, 256), 256, 0, s>>>(
          points, n, d, order.get(), nodeFirstTile.get(), nodeTileCount.get(), lb, le,
          split.get()); noteLaunch();
      levelKeysKernel<<<blocksFor(n, 256), 256, 0, s>>>(
          points, n, d, level, order.get(), nodeLeft.get(), nodeRight.get(), nodeFirstTile.get(),
          nodeTileCount.get(), split.get(), numInstances > 1 ? nodeSpans.get() : nullptr,
          keys.get()); noteLaunch();
      CUHC_TRY(st, cudaGetLastError());
      CUHC_TRY(st, cub::DeviceRadixSort::SortPairs(temp.get(), tempBytes, keys.get(),
                                                   keysOut.get(), order.get(), valsOut.get(), n,
                                                   0, 32 + tileBits, s));
      CUHC_TRY(st, cudaMemcpyAsync(order.get(), valsOut.get(), n * sizeof(int),
                                   cudaMemcpyDeviceToDevice, s));
    }
  }
  if (!st.ok())
    return st.code;
  CUHC_TRY(st, cudaMemsetAsync(tiled.get(), 0, tiled.bytes(), s));
  gatherTiledKernel<<<blocksFor(n, 128), 128, 0, s>>>(points, n, d, kc, numChunks, order.get(),
                                                      tiled.get(), rank.get()); noteLaunch();
  CUHC_TRY(st, cudaGetLastError());
  CUHC_TRY(st, retile(nullptr, n));
  return st.code;
}

int SpatialIndex::retile(const float *pointsByPosition, int newN) {
  normRangeKnown = false;
  StatusChain st;
  n = newN;
  if (pointsByPosition) {
    // Positions are the new slots; numTiles shrinks with n, topology follows.
    numTiles = numTilesFor(n);
    topo.build(numTiles);
    const int N = topo.numNodes;
    CUHC_TRY(st, cudaMemcpyAsync(nodeLeft.get(), topo.left.data(), N * sizeof(int),
                                 cudaMemcpyHostToDevice, stream));
    CUHC_TRY(st, cudaMemcpyAsync(nodeRight.get(), topo.right.data(), N * sizeof(int),
                                 cudaMemcpyHostToDevice, stream));
    CUHC_TRY(st, cudaMemcpyAsync(nodeFirstTile.get(), topo.firstTile.data(), N * sizeof(int),
                                 cudaMemcpyHostToDevice, stream));
    CUHC_TRY(st, cudaMemcpyAsync(nodeTileCount.get(), topo.tileCount.data(), N * sizeof(int),
                                 cudaMemcpyHostToDevice, stream));
    CUHC_TRY(st, cudaMemcpyAsync(leafOfTile.get(), topo.leafOfTile.data(),
                                 numTiles * sizeof(int), cudaMemcpyHostToDevice, stream));
    CUHC_TRY(st, cudaMemsetAsync(tiled.get(), 0, (size_t)numTiles * tileFloats() * sizeof(float),
                                 stream));
    gatherTiledKernel<<<blocksFor(n, 128), 128, 0, stream>>>(pointsByPosition, n, d, kc,
                                                             numChunks, nullptr, tiled.get(),
                                                             nullptr); noteLaunch();
    CUHC_TRY(st, cudaGetLastError());
  }
  const int N = topo.numNodes;
  leafBoxKernel<<<blocksFor((long long)numTiles * 32, 128), 128, 0, stream>>>(
      tiled.get(), n, d, kc, numChunks, numTiles, leafOfTile.get(),
      numInstances > 1 ? order.get() : nullptr, nodeLow.get(), nodeHigh.get()); noteLaunch();
  for (int level = topo.depth - 1; level >= 0; --level) {
    const int lb = topo.levelStart[level], le = topo.levelStart[level + 1];
    internalBoxKernel<<<blocksFor((long long)(le - lb) * d, 256), 256, 0, stream>>>(
        lb, le, d, nodeLeft.get(), nodeRight.get(), nodeLow.get(), nodeHigh.get()); noteLaunch();
  }
  (void)N;
  CUHC_TRY(st, cudaGetLastError());
  return st.code;
}

int SpatialIndex::updateMinValues(const float *values) {
  hasMinValues = values != nullptr;
  leafSummaryKernel<<<blocksFor((long long)numTiles * 32, 128), 128, 0, stream>>>(
      n, numTiles, leafOfTile.get(), values, nullptr, nodeMinValue.get(), nullptr); noteLaunch();
  for (int level = topo.depth - 1; level >= 0; --level) {
    const int lb = topo.levelStart[level], le = topo.levelStart[level + 1];
    internalSummaryKernel<<<blocksFor(le - lb, 128), 128, 0, stream>>>(
        lb, le, nodeLeft.get(), nodeRight.get(), nodeMinValue.get(), nullptr); noteLaunch();
  }
  return (int)cudaGetLastError();
}

bool SpatialIndex::extentsWithin(float limit) {
  std::vector<float> low(d), high(d);
  if (cudaMemcpyAsync(low.data(), nodeLow.get(), d * sizeof(float), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess ||
      cudaMemcpyAsync(high.data(), nodeHigh.get(), d * sizeof(float), cudaMemcpyDeviceToHost,
                      stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return false;
  for (int f = 0; f < d; ++f)
    if (!(high[f] - low[f] <= limit)) // NaN fails too
      return false;
  return true;
}

namespace {

// out[0] <- smallest nonzero squared norm, out[1] <- largest (float bits;
// squared norms are >= 0, so their bits order like the values), over the
// points of the tiled layout (padding slots skipped).
__global__ void normRange(const float *__restrict__ tiled, const int *__restrict__ order, int n,
                          int d, int kc, size_t tileFloats, unsigned int *__restrict__ out) {
  const int pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= n || order[pos] < 0)
    return;
  const float *tile = tiled + (size_t)(pos / kTile) * tileFloats;
  float sq = 0.0f;
  for (int k = 0; k < d; ++k) {
    const float x = tile[(size_t)((k / kc) * kc + k % kc) * kTile + pos % kTile];
    sq = fmaf(x, x, sq);
  }
  const unsigned int bits = __float_as_uint(sq);
  if (sq > 0.0f)
    atomicMin(out, bits);
  atomicMax(out + 1, bits);
}

} // namespace

bool SpatialIndex::normsWithin(float low, float high) {
  if (normRangeKnown)
    return normLow >= low && normHigh <= high;
  DeviceBuffer<unsigned int> range;
  unsigned int host[2] = {0x7f800000u, 0u};
  if (range.allocate(2, stream) != 0 ||
      cudaMemcpyAsync(range.get(), host, sizeof(host), cudaMemcpyHostToDevice, stream) !=
          cudaSuccess)
    return false;
  normRange<<<(n + 255) / 256, 256, 0, stream>>>(tiled.get(), order.get(), n, d, kc,
                                                 tileFloats(), range.get());
  noteLaunch();
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(host, range.get(), sizeof(host), cudaMemcpyDeviceToHost, stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return false;
  std::memcpy(&normLow, &host[0], sizeof(float));
  std::memcpy(&normHigh, &host[1], sizeof(float));
  normRangeKnown = true;
  // No nonzero point: the low end is +inf, which passes any bound.
  return normLow >= low && normHigh <= high;
}

namespace {

__global__ void tileKeysFromBoxes(const float *__restrict__ low, const float *__restrict__ high,
                                  const int *__restrict__ leafOfTile, int d, int numTiles,
                                  unsigned int *__restrict__ keys, int *__restrict__ iota) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= numTiles)
    return;
  const int node = leafOfTile[t];
  float score = 0.0f;
  for (int f = 0; f < d; ++f)
    score += __log2f(fmaxf(high[(size_t)node * d + f] - low[(size_t)node * d + f], 1e-30f));
  keys[t] = orderedBits(score);
  iota[t] = t;
}

__global__ void tileKeysFromWork(const unsigned int *__restrict__ work, int numTiles,
                                 const int *__restrict__ nodePure,
                                 const int *__restrict__ leafOfTile,
                                 unsigned int *__restrict__ keys, int *__restrict__ iota) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= numTiles)
    return;
  const unsigned int w = min(work[t], 0x7fffffffu);
  // Row tiles holding several components first (with nodePure): their rows
  // sit on component boundaries, where the components' lightest edges are.
  keys[t] = nodePure && nodePure[leafOfTile[t]] < 0 ? w | 0x80000000u : w;
  iota[t] = t;
}

} // namespace

int SpatialIndex::orderTiles(bool fromBoxes, bool impureFirst) {
  StatusChain st;
  if (!tileOrder.get()) {
    CUHC_TRY(st, tileWork.allocate(numTiles, stream));
    CUHC_TRY(st, tileOrder.allocate(numTiles, stream));
    CUHC_TRY(st, tileKeys.allocate(numTiles, stream));
    CUHC_TRY(st, tileKeysSorted.allocate(numTiles, stream));
    CUHC_TRY(st, tileIota.allocate(numTiles, stream));
    CUHC_TRY(st, cub::DeviceRadixSort::SortPairsDescending(
                     nullptr, tileSortBytes, tileKeys.get(), tileKeysSorted.get(), tileIota.get(),
                     tileOrder.get(), numTiles, 0, 32, stream));
    CUHC_TRY(st, tileSortTemp.allocate(std::max<size_t>(tileSortBytes, 1), stream));
    CUHC_TRY(st, cudaMemsetAsync(tileWork.get(), 0, numTiles * sizeof(unsigned int), stream));
    if (!st.ok())
      return st.code;
  }
  if (fromBoxes)
    tileKeysFromBoxes<<<blocksFor(numTiles, 256), 256, 0, stream>>>(
        nodeLow.get(), nodeHigh.get(), leafOfTile.get(), d, numTiles, tileKeys.get(),
        tileIota.get());
  else
    tileKeysFromWork<<<blocksFor(numTiles, 256), 256, 0, stream>>>(
        tileWork.get(), numTiles, impureFirst ? nodePure.get() : nullptr, leafOfTile.get(),
        tileKeys.get(), tileIota.get());
  noteLaunch();
  CUHC_TRY(st, cudaGetLastError());
  CUHC_TRY(st, cub::DeviceRadixSort::SortPairsDescending(
                   tileSortTemp.get(), tileSortBytes, tileKeys.get(), tileKeysSorted.get(),
                   tileIota.get(), tileOrder.get(), numTiles, 0, 32, stream));
  return st.code;
}

int SpatialIndex::updatePurity(const int *component) {
  leafSummaryKernel<<<blocksFor((long long)numTiles * 32, 128), 128, 0, stream>>>(
      n, numTiles, leafOfTile.get(), nullptr, component, nullptr, nodePure.get()); noteLaunch();
  for (int level = topo.depth - 1; level >= 0; --level) {
    const int lb = topo.levelStart[level], le = topo.levelStart[level + 1];
    internalSummaryKernel<<<blocksFor(le - lb, 128), 128, 0, stream>>>(
        lb, le, nodeLeft.get(), nodeRight.get(), nullptr, nodePure.get()); noteLaunch();
  }
  return (int)cudaGetLastError();
}

} // namespace cuhc

namespace cuhc {

int buildTiled(const float *points, int n, int d, DeviceBuffer<float> &tiled, cudaStream_t s) {
  const int kc = chunkWidthFor(d), numChunks = numChunksFor(d), T = numTilesFor(n);
  StatusChain st;
  CUHC_TRY(st, tiled.allocate((size_t)T * numChunks * kc * kTile, s));
  CUHC_TRY(st, cudaMemsetAsync(tiled.get(), 0, tiled.bytes(), s));
  if (!st.ok())
    return st.code;
  gatherTiledKernel<<<(n + 127) / 128, 128, 0, s>>>(points, n, d, kc, numChunks, nullptr,
                                                    tiled.get(), nullptr); noteLaunch();
  CUHC_TRY(st, cudaGetLastError());
  return st.code;
}

} // namespace cuhc
