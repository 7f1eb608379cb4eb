// The radius proposal's multilayer perceptron: 19 -> 64 -> 64 -> 1, ReLU,
// BF16 parameters and activations, FP32 accumulation (5,505 parameters).
//
// Parameter layout (FP32 master copy, `kMlpParams` floats):
//   W1 [19][64], b1 [64], W2 [64][64], b2 [64], w3 [64], b3 [1]
// The kernels round every parameter and every activation to BF16 (round to
// nearest even) before use, so forward results depend only on the BF16
// model, and accumulate each dot product in FP32 in index order.
//
// Forward: one thread per sample, parameters staged in shared memory as
// floats holding BF16 values. Backward (mean squared error on the output):
// each block takes kMlpBatch samples, keeps their activations and output
// gradients in shared memory, and forms the parameter gradients as the
// block's small products (dW2 = H1^T D2 etc.), every thread owning a slice
// of the outputs; one atomicAdd per parameter per block. Adam updates the
// FP32 master parameters.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include <atomic>
#include <mutex>

#include "common.cuh"
#include "profiling.cuh"
#include "radius.cuh"

namespace cuhc {

constexpr int kMlpIn = 19, kMlpHidden = 64;
constexpr int kW1 = 0, kB1 = kW1 + kMlpIn * kMlpHidden, kW2 = kB1 + kMlpHidden,
              kB2 = kW2 + kMlpHidden * kMlpHidden, kW3 = kB2 + kMlpHidden, kB3 = kW3 + kMlpHidden;
constexpr int kMlpParams = kB3 + 1; // 5,505
constexpr int kMlpBatch = 128;      // samples per block in the backward kernel

__device__ __forceinline__ float bf16(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Parameters rounded to BF16 into shared memory.
__device__ __forceinline__ void stageParams(const float *__restrict__ params, float *sp) {
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x)
    sp[i] = bf16(params[i]);
  __syncthreads();
}

// Forward of one sample from BF16 parameters sp; activations to h1, h2.
__device__ __forceinline__ float forwardOne(const float *sp, const float *x, float *h1,
                                            float *h2) {
  float xin[kMlpIn];
#pragma unroll
  for (int i = 0; i < kMlpIn; ++i)
    xin[i] = bf16(x[i]);
  for (int j = 0; j < kMlpHidden; ++j) {
    float a = 0.0f;
#pragma unroll
    for (int i = 0; i < kMlpIn; ++i)
      a = fmaf(xin[i], sp[kW1 + i * kMlpHidden + j], a);
    h1[j] = bf16(fmaxf(a + sp[kB1 + j], 0.0f));
  }
  for (int k = 0; k < kMlpHidden; ++k) {
    float a = 0.0f;
    for (int j = 0; j < kMlpHidden; ++j)
      a = fmaf(h1[j], sp[kW2 + j * kMlpHidden + k], a);
    h2[k] = bf16(fmaxf(a + sp[kB2 + k], 0.0f));
  }
  float out = 0.0f;
  for (int k = 0; k < kMlpHidden; ++k)
    out = fmaf(h2[k], sp[kW3 + k], out);
  return out + sp[kB3];
}

static __global__ void __launch_bounds__(128)
    mlpForwardKernel(const float *__restrict__ params, const float *__restrict__ x, int count,
                     float *__restrict__ out) {
  __shared__ float sp[kMlpParams];
  stageParams(params, sp);
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= count)
    return;
  float h1[kMlpHidden], h2[kMlpHidden];
  out[s] = forwardOne(sp, x + (size_t)s * kMlpIn, h1, h2);
}

// Gradient of L = sum over samples of (out - y)^2 / count, added into grad;
// loss receives the summed squared error.
static __global__ void __launch_bounds__(kMlpBatch)
    mlpGradientKernel(const float *__restrict__ params, const float *__restrict__ x,
                      const float *__restrict__ y, int count, float *__restrict__ grad,
                      float *__restrict__ loss) {
  extern __shared__ float dyn[];
  float *sp = dyn;                               // kMlpParams
  float *sx = sp + kMlpParams;                   // [batch][19]
  float *sh1 = sx + kMlpBatch * kMlpIn;          // [batch][64]
  float *sh2 = sh1 + kMlpBatch * kMlpHidden;     // [batch][64]
  float *sd2 = sh2 + kMlpBatch * kMlpHidden;     // [batch][64]: dL/d(pre-activation 2)
  float *sd1 = sd2 + kMlpBatch * kMlpHidden;     // [batch][64]: dL/d(pre-activation 1)
  float *sdo = sd1 + kMlpBatch * kMlpHidden;     // [batch]: dL/d(out)
  stageParams(params, sp);
  const int t = threadIdx.x;
  const int s = blockIdx.x * kMlpBatch + t;
  const bool valid = s < count;
  float h1[kMlpHidden], h2[kMlpHidden];
  float d2[kMlpHidden];
  if (valid) {
    for (int i = 0; i < kMlpIn; ++i)
      sx[t * kMlpIn + i] = bf16(x[(size_t)s * kMlpIn + i]);
    const float out = forwardOne(sp, x + (size_t)s * kMlpIn, h1, h2);
    const float err = out - y[s];
    atomicAdd(loss, err * err);
    const float dout = 2.0f * err / (float)count;
    sdo[t] = dout;
    for (int k = 0; k < kMlpHidden; ++k) {
      sh1[t * kMlpHidden + k] = h1[k];
      sh2[t * kMlpHidden + k] = h2[k];
      d2[k] = h2[k] > 0.0f ? dout * sp[kW3 + k] : 0.0f;
      sd2[t * kMlpHidden + k] = d2[k];
    }
    for (int j = 0; j < kMlpHidden; ++j) {
      float a = 0.0f;
      for (int k = 0; k < kMlpHidden; ++k)
        a = fmaf(d2[k], sp[kW2 + j * kMlpHidden + k], a);
      sd1[t * kMlpHidden + j] = h1[j] > 0.0f ? a : 0.0f;
    }
  } else {
    for (int i = 0; i < kMlpIn; ++i)
      sx[t * kMlpIn + i] = 0.0f;
    sdo[t] = 0.0f;
    for (int k = 0; k < kMlpHidden; ++k)
      sh1[t * kMlpHidden + k] = sh2[t * kMlpHidden + k] = sd2[t * kMlpHidden + k] =
          sd1[t * kMlpHidden + k] = 0.0f;
  }
  __syncthreads();
  // Block products over the batch; thread t owns parameters t, t + 128, ...
  for (int q = t; q < kMlpParams; q += kMlpBatch) {
    float g = 0.0f;
    if (q < kB1) {
      const int i = q / kMlpHidden, j = q % kMlpHidden;
      for (int b = 0; b < kMlpBatch; ++b)
        g = fmaf(sx[b * kMlpIn + i], sd1[b * kMlpHidden + j], g);
    } else if (q < kW2) {
      const int j = q - kB1;
      for (int b = 0; b < kMlpBatch; ++b)
        g += sd1[b * kMlpHidden + j];
    } else if (q < kB2) {
      const int j = (q - kW2) / kMlpHidden, k = (q - kW2) % kMlpHidden;
      for (int b = 0; b < kMlpBatch; ++b)
        g = fmaf(sh1[b * kMlpHidden + j], sd2[b * kMlpHidden + k], g);
    } else if (q < kW3) {
      const int k = q - kB2;
      for (int b = 0; b < kMlpBatch; ++b)
        g += sd2[b * kMlpHidden + k];
    } else if (q < kB3) {
      const int k = q - kW3;
      for (int b = 0; b < kMlpBatch; ++b)
        g = fmaf(sh2[b * kMlpHidden + k], sdo[b], g);
    } else {
      for (int b = 0; b < kMlpBatch; ++b)
        g += sdo[b];
    }
    atomicAdd(grad + q, g);
  }
}

static __global__ void adamKernel(float *__restrict__ params, const float *__restrict__ grad,
                                  float *__restrict__ m1, float *__restrict__ m2, float lr,
                                  float beta1, float beta2, float correction1,
                                  float correction2) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= kMlpParams)
    return;
  const float g = grad[q];
  m1[q] = beta1 * m1[q] + (1.0f - beta1) * g;
  m2[q] = beta2 * m2[q] + (1.0f - beta2) * g * g;
  const float mh = m1[q] / correction1, vh = m2[q] / correction2;
  params[q] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

size_t mlpGradientShared() {
  return ((size_t)kMlpParams + kMlpBatch * (kMlpIn + 4 * kMlpHidden + 1)) * sizeof(float);
}

int mlpForward(const float *params, const float *x, int count, float *out, cudaStream_t s) {
  if (count <= 0)
    return 0;
  mlpForwardKernel<<<(count + 127) / 128, 128, 0, s>>>(params, x, count, out);
  noteLaunch();
  return (int)cudaGetLastError();
}

int mlpGradient(const float *params, const float *x, const float *y, int count, float *grad,
                float *loss, cudaStream_t s) {
  StatusChain st;
  CUHC_TRY(st, cudaMemsetAsync(grad, 0, kMlpParams * sizeof(float), s));
  CUHC_TRY(st, cudaMemsetAsync(loss, 0, sizeof(float), s));
  if (count <= 0 || !st.ok())
    return st.code;
  const size_t shared = mlpGradientShared();
  CUHC_TRY(st, cudaFuncSetAttribute(mlpGradientKernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)shared));
  mlpGradientKernel<<<(count + kMlpBatch - 1) / kMlpBatch, kMlpBatch, shared, s>>>(
      params, x, y, count, grad, loss);
  noteLaunch();
  CUHC_TRY(st, cudaGetLastError());
  return st.code;
}

// The radius model: one device copy per device that used it, made on first
// use after cuhc_set_radius_model.
namespace {
std::mutex gModelMutex;
std::vector<float> gModelHost;
float gModelOffset = 0.0f;
unsigned long long gModelVersion = 0;
constexpr int kMaxDevices = 64;
float *gModelDevice[kMaxDevices] = {};
unsigned long long gModelDeviceVersion[kMaxDevices] = {};
std::atomic<unsigned long long> gRadiusProposed{0}, gRadiusCertified{0}, gRadiusCappedTiles{0},
    gRadiusFallbackTiles{0};
} // namespace

RadiusModel currentRadiusModel() {
  std::lock_guard<std::mutex> lock(gModelMutex);
  RadiusModel model;
  if (gModelHost.empty())
    return model;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices)
    return model;
  if (gModelDeviceVersion[device] != gModelVersion) {
    if (!gModelDevice[device] &&
        cudaMalloc(&gModelDevice[device], kMlpParams * sizeof(float)) != cudaSuccess) {
      gModelDevice[device] = nullptr;
      return model;
    }
    if (cudaMemcpy(gModelDevice[device], gModelHost.data(), kMlpParams * sizeof(float),
                   cudaMemcpyHostToDevice) != cudaSuccess)
      return model;
    gModelDeviceVersion[device] = gModelVersion;
  }
  model.params = gModelDevice[device];
  model.offset = gModelOffset;
  return model;
}

void addRadiusStats(unsigned long long proposed, unsigned long long certified,
                    unsigned long long cappedTiles, unsigned long long fallbackTiles) {
  gRadiusProposed += proposed;
  gRadiusCertified += certified;
  gRadiusCappedTiles += cappedTiles;
  gRadiusFallbackTiles += fallbackTiles;
}

} // namespace cuhc

using namespace cuhc;

extern "C" {

// Loads the radius proposal's model (5,505 floats, host) with its calibration
// offset; params NULL switches the proposal off. Results never change.
int cuhc_set_radius_model(const float *params, float offset) {
  std::lock_guard<std::mutex> lock(gModelMutex);
  if (params)
    gModelHost.assign(params, params + kMlpParams);
  else
    gModelHost.clear();
  gModelOffset = offset;
  ++gModelVersion;
  return 0;
}

// Since the last call (first `count` of the four; resets them): rows given a
// proposed radius, rows the capped pass certified, tiles the capped passes
// computed, tiles the fallback passes computed.
int cuhc_radius_stats(unsigned long long *out, int count) {
  const unsigned long long v[4] = {gRadiusProposed.exchange(0), gRadiusCertified.exchange(0),
                                   gRadiusCappedTiles.exchange(0),
                                   gRadiusFallbackTiles.exchange(0)};
  for (int i = 0; i < count && i < 4; ++i)
    out[i] = v[i];
  return 0;
}

// Forward of the radius MLP on HOST buffers: params (5,505 floats, the layout
// above), x [count][19], out [count]. No counterpart in the reference.
int cuhc_mlp_forward(const float *params, const float *x, int count, float *out) {
  if (count < 0)
    return kErrorInvalidShape;
  StatusChain st;
  DeviceBuffer<float> dp, dx, dout;
  CUHC_TRY(st, dp.allocate(kMlpParams, 0));
  CUHC_TRY(st, dx.allocate((size_t)std::max(count, 1) * kMlpIn, 0));
  CUHC_TRY(st, dout.allocate(std::max(count, 1), 0));
  CUHC_TRY(st, cudaMemcpyAsync(dp.get(), params, kMlpParams * sizeof(float),
                               cudaMemcpyHostToDevice, 0));
  CUHC_TRY(st, cudaMemcpyAsync(dx.get(), x, (size_t)count * kMlpIn * sizeof(float),
                               cudaMemcpyHostToDevice, 0));
  CUHC_TRY(st, mlpForward(dp.get(), dx.get(), count, dout.get(), 0));
  CUHC_TRY(st, cudaMemcpyAsync(out, dout.get(), (size_t)count * sizeof(float),
                               cudaMemcpyDeviceToHost, 0));
  CUHC_TRY(st, cudaStreamSynchronize(0));
  return st.code;
}

// Gradient of the mean squared error over the samples (host buffers);
// loss receives the mean squared error.
int cuhc_mlp_gradient(const float *params, const float *x, const float *y, int count, float *grad,
                      float *loss) {
  if (count < 1)
    return kErrorInvalidShape;
  StatusChain st;
  DeviceBuffer<float> dp, dx, dy, dg, dl;
  CUHC_TRY(st, dp.allocate(kMlpParams, 0));
  CUHC_TRY(st, dx.allocate((size_t)count * kMlpIn, 0));
  CUHC_TRY(st, dy.allocate(count, 0));
  CUHC_TRY(st, dg.allocate(kMlpParams, 0));
  CUHC_TRY(st, dl.allocate(1, 0));
  CUHC_TRY(st, cudaMemcpyAsync(dp.get(), params, kMlpParams * sizeof(float),
                               cudaMemcpyHostToDevice, 0));
  CUHC_TRY(st, cudaMemcpyAsync(dx.get(), x, (size_t)count * kMlpIn * sizeof(float),
                               cudaMemcpyHostToDevice, 0));
  CUHC_TRY(st, cudaMemcpyAsync(dy.get(), y, (size_t)count * sizeof(float),
                               cudaMemcpyHostToDevice, 0));
  CUHC_TRY(st, mlpGradient(dp.get(), dx.get(), dy.get(), count, dg.get(), dl.get(), 0));
  float sum = 0.0f;
  CUHC_TRY(st, cudaMemcpyAsync(grad, dg.get(), kMlpParams * sizeof(float),
                               cudaMemcpyDeviceToHost, 0));
  CUHC_TRY(st, cudaMemcpyAsync(&sum, dl.get(), sizeof(float), cudaMemcpyDeviceToHost, 0));
  CUHC_TRY(st, cudaStreamSynchronize(0));
  if (loss)
    *loss = sum / (float)count;
  return st.code;
}

// Adam on the GPU: `epochs` passes over the samples in shuffled minibatches
// of `batch` (seeded), learning rate lr; params (host, 5,505 floats) in/out;
// losses (may be NULL) receives each epoch's mean squared error.
int cuhc_mlp_train(const float *x, const float *y, int count, int epochs, int batch, float lr,
                   unsigned long long seed, float *params, float *losses) {
  if (count < 1 || epochs < 0 || batch < 1)
    return kErrorInvalidShape;
  StatusChain st;
  DeviceBuffer<float> dp, dx, dy, dg, dl, m1, m2, bx, by;
  CUHC_TRY(st, dp.allocate(kMlpParams, 0));
  CUHC_TRY(st, dx.allocate((size_t)count * kMlpIn, 0));
  CUHC_TRY(st, dy.allocate(count, 0));
  CUHC_TRY(st, dg.allocate(kMlpParams, 0));
  CUHC_TRY(st, dl.allocate(1, 0));
  CUHC_TRY(st, m1.allocate(kMlpParams, 0));
  CUHC_TRY(st, m2.allocate(kMlpParams, 0));
  CUHC_TRY(st, bx.allocate((size_t)batch * kMlpIn, 0));
  CUHC_TRY(st, by.allocate(batch, 0));
  CUHC_TRY(st, cudaMemcpyAsync(dp.get(), params, kMlpParams * sizeof(float),
                               cudaMemcpyHostToDevice, 0));
  CUHC_TRY(st, cudaMemsetAsync(m1.get(), 0, kMlpParams * sizeof(float), 0));
  CUHC_TRY(st, cudaMemsetAsync(m2.get(), 0, kMlpParams * sizeof(float), 0));
  // Minibatches are gathered on the host (a seeded shuffle per epoch).
  std::vector<int> perm(count);
  for (int i = 0; i < count; ++i)
    perm[i] = i;
  std::vector<float> hx((size_t)batch * kMlpIn), hy(batch);
  unsigned long long state = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto next = [&]() {
    state = state * 6364136223846793005ull + 1442695040888963407ull;
    return (uint32_t)(state >> 33);
  };
  int step = 0;
  const float beta1 = 0.9f, beta2 = 0.999f;
  for (int e = 0; e < epochs && st.ok(); ++e) {
    for (int i = count - 1; i > 0; --i)
      std::swap(perm[i], perm[next() % (uint32_t)(i + 1)]);
    double epochLoss = 0.0;
    for (int start = 0; start < count && st.ok(); start += batch) {
      const int m = std::min(batch, count - start);
      for (int b = 0; b < m; ++b) {
        const int src = perm[start + b];
        for (int f = 0; f < kMlpIn; ++f)
          hx[(size_t)b * kMlpIn + f] = x[(size_t)src * kMlpIn + f];
        hy[b] = y[src];
      }
      CUHC_TRY(st, cudaMemcpyAsync(bx.get(), hx.data(), (size_t)m * kMlpIn * sizeof(float),
                                   cudaMemcpyHostToDevice, 0));
      CUHC_TRY(st, cudaMemcpyAsync(by.get(), hy.data(), (size_t)m * sizeof(float),
                                   cudaMemcpyHostToDevice, 0));
      CUHC_TRY(st, mlpGradient(dp.get(), bx.get(), by.get(), m, dg.get(), dl.get(), 0));
      ++step;
      adamKernel<<<(kMlpParams + 255) / 256, 256, 0, 0>>>(
          dp.get(), dg.get(), m1.get(), m2.get(), lr, beta1, beta2,
          1.0f - std::pow(beta1, (float)step), 1.0f - std::pow(beta2, (float)step));
      noteLaunch();
      CUHC_TRY(st, cudaGetLastError());
      float sum = 0.0f;
      CUHC_TRY(st, cudaMemcpyAsync(&sum, dl.get(), sizeof(float), cudaMemcpyDeviceToHost, 0));
      CUHC_TRY(st, cudaStreamSynchronize(0)); // hx / hy are reused next minibatch
      epochLoss += sum;
    }
    if (losses)
      losses[e] = (float)(epochLoss / count);
  }
  CUHC_TRY(st, cudaMemcpyAsync(params, dp.get(), kMlpParams * sizeof(float),
                               cudaMemcpyDeviceToHost, 0));
  CUHC_TRY(st, cudaStreamSynchronize(0));
  return st.code;
}

} // extern "C"
