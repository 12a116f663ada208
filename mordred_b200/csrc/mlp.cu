// mlp.cu — the learned planner's cost model: a 24 -> 64 -> 64 -> 2 ReLU MLP (5,890
// fp32 parameters) that maps a (query, segment) feature vector to the predicted log CPU
// ms and log GPU ms of running the segment on each device. Forward, backward and Adam
// are hand-written kernels; the reference plans with an analytic bandwidth model
// instead (src/gpudb/CostModel.cu:283-440), which stays as the fallback.
//
// Parameter layout (one flat fp32 array): W1[24][64], b1[64], W2[64][64], b2[64],
// W3[64][2], b3[2]; W[i][j] is input i -> unit j. A block takes a tile of kTile samples:
// the tile's inputs and both hidden layers sit in shared memory, each thread computes
// some (sample, unit) dot products. The backward kernel recomputes the forward pass of
// its tile, forms dL/dy = (y - t) / B for the loss 1/(2B) * sum (y - t)^2, propagates it
// through the ReLUs, and adds the tile's weight gradients into the global gradient with
// fp32 atomics (so summation order, and the last bits, vary from run to run).
// SIMT fp32 on purpose: 11.5 kFLOP per sample is far too small for tensor cores to pay.
#include <cmath>

#include "common.cuh"

namespace mb {

constexpr int kIn = MB_MLP_IN, kHid = MB_MLP_HIDDEN, kOut = MB_MLP_OUT;
constexpr int kW1 = 0, kB1 = kW1 + kIn * kHid, kW2 = kB1 + kHid, kB2 = kW2 + kHid * kHid, kW3 = kB2 + kHid,
              kB3 = kW3 + kHid * kOut, kParams = kB3 + kOut;
static_assert(kParams == MB_MLP_PARAMS, "parameter count");
constexpr int kTile = 32;
constexpr int kThreads = 256;

struct MlpSmem {
  float w[kParams];
  float x[kTile][kIn];
  float h1[kTile][kHid];
  float h2[kTile][kHid];
  float dy[kTile][kOut];
  float d2[kTile][kHid];
  float d1[kTile][kHid];
};

// Forward pass of rows [r0, r0 + nt) into s.h1, s.h2; returns nothing, outputs via `out`.
__device__ void tile_forward(MlpSmem& s, const float* x, int r0, int nt, float* out) {
  const int tid = threadIdx.x;
  for (int i = tid; i < kTile * kIn; i += kThreads) {
    const int b = i / kIn, k = i % kIn;
    s.x[b][k] = b < nt ? x[static_cast<long long>(r0 + b) * kIn + k] : 0.f;
  }
  __syncthreads();
  for (int i = tid; i < kTile * kHid; i += kThreads) {
    const int b = i / kHid, j = i % kHid;
    float a = s.w[kB1 + j];
#pragma unroll 8
    for (int k = 0; k < kIn; ++k) a = fmaf(s.x[b][k], s.w[kW1 + k * kHid + j], a);
    s.h1[b][j] = fmaxf(a, 0.f);
  }
  __syncthreads();
  for (int i = tid; i < kTile * kHid; i += kThreads) {
    const int b = i / kHid, j = i % kHid;
    float a = s.w[kB2 + j];
#pragma unroll 8
    for (int k = 0; k < kHid; ++k) a = fmaf(s.h1[b][k], s.w[kW2 + k * kHid + j], a);
    s.h2[b][j] = fmaxf(a, 0.f);
  }
  __syncthreads();
  for (int i = tid; i < kTile * kOut; i += kThreads) {
    const int b = i / kOut, o = i % kOut;
    float a = s.w[kB3 + o];
#pragma unroll 8
    for (int k = 0; k < kHid; ++k) a = fmaf(s.h2[b][k], s.w[kW3 + k * kOut + o], a);
    out[i] = a;  // caller-provided per-tile buffer (shared)
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kThreads) mlp_forward_kernel(const float* __restrict__ params,
                                                               const float* __restrict__ x, int batch,
                                                               float* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char raw[];
  MlpSmem& s = *reinterpret_cast<MlpSmem*>(raw);
  for (int i = threadIdx.x; i < kParams; i += kThreads) s.w[i] = params[i];
  for (int r0 = blockIdx.x * kTile; r0 < batch; r0 += gridDim.x * kTile) {
    const int nt = min(kTile, batch - r0);
    __syncthreads();
    tile_forward(s, x, r0, nt, &s.dy[0][0]);
    for (int i = threadIdx.x; i < nt * kOut; i += kThreads) y[static_cast<long long>(r0) * kOut + i] = (&s.dy[0][0])[i];
  }
}

__global__ void __launch_bounds__(kThreads) mlp_backward_kernel(const float* __restrict__ params,
                                                                const float* __restrict__ x,
                                                                const float* __restrict__ target, int batch,
                                                                float* __restrict__ grads, float* loss_sum) {
  extern __shared__ __align__(16) unsigned char raw[];
  MlpSmem& s = *reinterpret_cast<MlpSmem*>(raw);
  const int tid = threadIdx.x;
  for (int i = tid; i < kParams; i += kThreads) s.w[i] = params[i];
  const float inv_b = 1.f / static_cast<float>(batch);
  for (int r0 = blockIdx.x * kTile; r0 < batch; r0 += gridDim.x * kTile) {
    const int nt = min(kTile, batch - r0);
    __syncthreads();
    tile_forward(s, x, r0, nt, &s.dy[0][0]);
    // dL/dy and the loss
    float part = 0.f;
    for (int i = tid; i < kTile * kOut; i += kThreads) {
      const int b = i / kOut;
      float d = 0.f;
      if (b < nt) {
        d = (&s.dy[0][0])[i] - target[static_cast<long long>(r0) * kOut + i];
        part += d * d;
      }
      (&s.dy[0][0])[i] = d * inv_b;
    }
    if (loss_sum) {
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
      if ((tid & 31) == 0 && part != 0.f) atomicAdd(loss_sum, 0.5f * part);
    }
    __syncthreads();
    // dL/dh2 (through the second ReLU)
    for (int i = tid; i < kTile * kHid; i += kThreads) {
      const int b = i / kHid, j = i % kHid;
      float a = 0.f;
#pragma unroll
      for (int o = 0; o < kOut; ++o) a = fmaf(s.dy[b][o], s.w[kW3 + j * kOut + o], a);
      s.d2[b][j] = s.h2[b][j] > 0.f ? a : 0.f;
    }
    __syncthreads();
    // dL/dh1 (through the first ReLU)
    for (int i = tid; i < kTile * kHid; i += kThreads) {
      const int b = i / kHid, k = i % kHid;
      float a = 0.f;
#pragma unroll 8
      for (int j = 0; j < kHid; ++j) a = fmaf(s.d2[b][j], s.w[kW2 + k * kHid + j], a);
      s.d1[b][k] = s.h1[b][k] > 0.f ? a : 0.f;
    }
    __syncthreads();
    // weight gradients of the tile: each thread sums its entries over the tile's samples
    for (int i = tid; i < kParams; i += kThreads) {
      float g = 0.f;
      if (i < kB1) {
        const int k = i / kHid, j = i % kHid;
        for (int b = 0; b < nt; ++b) g = fmaf(s.x[b][k], s.d1[b][j], g);
      } else if (i < kW2) {
        const int j = i - kB1;
        for (int b = 0; b < nt; ++b) g += s.d1[b][j];
      } else if (i < kB2) {
        const int k = (i - kW2) / kHid, j = (i - kW2) % kHid;
        for (int b = 0; b < nt; ++b) g = fmaf(s.h1[b][k], s.d2[b][j], g);
      } else if (i < kW3) {
        const int j = i - kB2;
        for (int b = 0; b < nt; ++b) g += s.d2[b][j];
      } else if (i < kB3) {
        const int k = (i - kW3) / kOut, o = (i - kW3) % kOut;
        for (int b = 0; b < nt; ++b) g = fmaf(s.h2[b][k], s.dy[b][o], g);
      } else {
        const int o = i - kB3;
        for (int b = 0; b < nt; ++b) g += s.dy[b][o];
      }
      if (g != 0.f) atomicAdd(grads + i, g);
    }
  }
}

__global__ void mlp_adam_kernel(float* __restrict__ params, const float* __restrict__ grads, float* __restrict__ m,
                                float* __restrict__ v, int n, float lr, float beta1, float beta2, float eps,
                                float bc1, float bc2, float weight_decay) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float g = grads[i] + weight_decay * params[i];
    const float mi = beta1 * m[i] + (1.f - beta1) * g;
    const float vi = beta2 * v[i] + (1.f - beta2) * g * g;
    m[i] = mi;
    v[i] = vi;
    params[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}

static int mlp_grid(long long batch) {
  int err = MB_OK;
  DeviceState* ds = current_device_state(&err);
  const int sms = ds ? ds->num_sms : 148;
  long long tiles = (batch + kTile - 1) / kTile;
  return static_cast<int>(tiles < sms ? tiles : sms);
}

// The tile needs more than the default 48 KB of shared memory: opt in (on the current device).
static bool mlp_init_attrs() {
  const int bytes = static_cast<int>(sizeof(MlpSmem));
  if (cudaFuncSetAttribute(reinterpret_cast<const void*>(mlp_forward_kernel),
                           cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess ||
      cudaFuncSetAttribute(reinterpret_cast<const void*>(mlp_backward_kernel),
                           cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
    return false;
  return true;
}

}  // namespace mb

using namespace mb;

extern "C" int mb_mlp_forward(const float* params, const float* x, int batch, float* y, mb_stream_t stream) {
  if (batch == 0) return MB_OK;
  if (params == nullptr || x == nullptr || y == nullptr || batch < 0) return MB_ERR_ARG;
  int err = MB_OK;
  if (current_device_state(&err) == nullptr) return err;
  if (!mlp_init_attrs()) return MB_ERR_CUDA;
  mlp_forward_kernel<<<mlp_grid(batch), kThreads, sizeof(MlpSmem), static_cast<cudaStream_t>(stream)>>>(params, x,
                                                                                                       batch, y);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);
  return MB_OK;
}

extern "C" int mb_mlp_backward(const float* params, const float* x, const float* target, int batch, float* grads,
                               float* loss_sum, mb_stream_t stream) {
  if (batch == 0) return MB_OK;
  if (params == nullptr || x == nullptr || target == nullptr || grads == nullptr || batch < 0) return MB_ERR_ARG;
  int err = MB_OK;
  if (current_device_state(&err) == nullptr) return err;
  if (!mlp_init_attrs()) return MB_ERR_CUDA;
  mlp_backward_kernel<<<mlp_grid(batch), kThreads, sizeof(MlpSmem), static_cast<cudaStream_t>(stream)>>>(
      params, x, target, batch, grads, loss_sum);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);
  return MB_OK;
}

extern "C" int mb_mlp_adam(float* params, const float* grads, float* m, float* v, int n, float lr, float beta1,
                           float beta2, float eps, int step, float weight_decay, mb_stream_t stream) {
  if (n == 0) return MB_OK;
  if (params == nullptr || grads == nullptr || m == nullptr || v == nullptr || n < 0 || step < 1) return MB_ERR_ARG;
  // bias corrections 1 - beta^step, computed on the host in double
  const float bc1 = static_cast<float>(1.0 - std::pow(static_cast<double>(beta1), step));
  const float bc2 = static_cast<float>(1.0 - std::pow(static_cast<double>(beta2), step));
  int blocks = (n + 255) / 256;
  if (blocks > 1024) blocks = 1024;
  mlp_adam_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(params, grads, m, v, n, lr, beta1, beta2,
                                                                         eps, bc1, bc2, weight_decay);
  if (cudaGetLastError() != cudaSuccess) return MB_ERR_LAUNCH;
  note_launches(1);
  return MB_OK;
}
