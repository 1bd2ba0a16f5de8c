// Training kernels of the T5 classifier (SDL/NeuralNetwork.h: 38 inputs ->
// 32 ReLU -> 32 ReLU -> 1, sigmoid on the output).  The inference copy lives
// in the quintuplet kernels; these are the forward pass that keeps the hidden
// activations and the backward (adjoint) pass that turns the loss gradient
// w.r.t. the logits into the gradient w.r.t. all 2337 parameters.
//
// Parameter layout (as the weight file): W0[38][32], b0[32], W2[32][32],
// b2[32], w4[32], b4.  The weight gradients are sums over samples; they are
// formed as fixed-order partial sums over chunks of samples followed by a
// fixed-order sum of the chunks, so the result does not depend on scheduling.
#include <cuda_runtime.h>

#include <string>

#include "lst_b200.h"

namespace {

  constexpr int kIn = 38, kH = 32;
  constexpr int kW0 = 0, kB0 = kIn * kH, kW2 = kB0 + kH, kB2 = kW2 + kH * kH, kW4 = kB2 + kH, kB4 = kW4 + kH;
  constexpr int kParams = kB4 + 1;
  static_assert(kParams == 2337, "T5 DNN parameter count");
  constexpr int kChunk = 256;  // samples per partial gradient sum

  __global__ void kDnnForward(const float* __restrict__ W, const float* __restrict__ x, int n, float* __restrict__ h1,
                              float* __restrict__ h2, float* __restrict__ logit) {
    __shared__ float sW[kParams];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x)
      sW[i] = W[i];
    __syncthreads();
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
      float xi[kIn];
#pragma unroll
      for (int k = 0; k < kIn; ++k)
        xi[k] = x[size_t(s) * kIn + k];
      float a1[kH];
#pragma unroll
      for (int c = 0; c < kH; ++c) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < kIn; ++k)
          acc += xi[k] * sW[kW0 + k * kH + c];
        acc += sW[kB0 + c];
        a1[c] = acc > 0.f ? acc : 0.f;
        h1[size_t(s) * kH + c] = a1[c];
      }
      float z = 0.f;
#pragma unroll
      for (int c = 0; c < kH; ++c) {
        float acc = 0.f;
#pragma unroll
        for (int k = 0; k < kH; ++k)
          acc += a1[k] * sW[kW2 + k * kH + c];
        acc += sW[kB2 + c];
        const float a2 = acc > 0.f ? acc : 0.f;
        h2[size_t(s) * kH + c] = a2;
        z += a2 * sW[kW4 + c];
      }
      logit[s] = z + sW[kB4];
    }
  }

  // Per sample: dh2 = dz * w4 (ReLU-gated), dh1 = W2 dh2 (ReLU-gated).
  __global__ void kDnnBackSample(const float* __restrict__ W, const float* __restrict__ h1, const float* __restrict__ h2,
                                 const float* __restrict__ dlogit, int n, float* __restrict__ dh1,
                                 float* __restrict__ dh2) {
    __shared__ float sW[kParams];
    for (int i = threadIdx.x; i < kParams; i += blockDim.x)
      sW[i] = W[i];
    __syncthreads();
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
      const float dz = dlogit[s];
      float g2[kH];
#pragma unroll
      for (int j = 0; j < kH; ++j) {
        g2[j] = h2[size_t(s) * kH + j] > 0.f ? dz * sW[kW4 + j] : 0.f;
        dh2[size_t(s) * kH + j] = g2[j];
      }
#pragma unroll
      for (int i = 0; i < kH; ++i) {
        float acc = 0.f;
#pragma unroll
        for (int j = 0; j < kH; ++j)
          acc += g2[j] * sW[kW2 + i * kH + j];
        dh1[size_t(s) * kH + i] = h1[size_t(s) * kH + i] > 0.f ? acc : 0.f;
      }
    }
  }

  // partial[chunk][g] = sum over the chunk's samples of gradient element g.
  __global__ void kDnnGradPartial(const float* __restrict__ x, const float* __restrict__ h1, const float* __restrict__ h2,
                                  const float* __restrict__ dlogit, const float* __restrict__ dh1,
                                  const float* __restrict__ dh2, int n, float* __restrict__ partial) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int chunk = blockIdx.y;
    if (g >= kParams)
      return;
    const int s0 = chunk * kChunk;
    const int s1 = min(n, s0 + kChunk);
    float acc = 0.f;
    if (g < kB0) {  // W0[k][i]: x[s][k] * dh1[s][i]
      const int k = g / kH, i = g % kH;
      for (int s = s0; s < s1; ++s)
        acc += x[size_t(s) * kIn + k] * dh1[size_t(s) * kH + i];
    } else if (g < kW2) {  // b0[i]
      const int i = g - kB0;
      for (int s = s0; s < s1; ++s)
        acc += dh1[size_t(s) * kH + i];
    } else if (g < kB2) {  // W2[i][j]: h1[s][i] * dh2[s][j]
      const int i = (g - kW2) / kH, j = (g - kW2) % kH;
      for (int s = s0; s < s1; ++s)
        acc += h1[size_t(s) * kH + i] * dh2[size_t(s) * kH + j];
    } else if (g < kW4) {  // b2[j]
      const int j = g - kB2;
      for (int s = s0; s < s1; ++s)
        acc += dh2[size_t(s) * kH + j];
    } else if (g < kB4) {  // w4[j]: h2[s][j] * dz[s]
      const int j = g - kW4;
      for (int s = s0; s < s1; ++s)
        acc += h2[size_t(s) * kH + j] * dlogit[s];
    } else {  // b4
      for (int s = s0; s < s1; ++s)
        acc += dlogit[s];
    }
    partial[size_t(chunk) * kParams + g] = acc;
  }

  __global__ void kDnnGradReduce(const float* __restrict__ partial, int nChunks, float* __restrict__ grad) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= kParams)
      return;
    float acc = 0.f;
    for (int c = 0; c < nChunks; ++c)
      acc += partial[size_t(c) * kParams + g];
    grad[g] = acc;
  }

  thread_local std::string g_dnnError;

  int dnnFail(const char* what) {
    cudaError_t e = cudaGetLastError();
    g_dnnError = std::string(what) + ": " + cudaGetErrorString(e);
    return -1;
  }

  int blocksFor(int n, int threads) {
    int b = (n + threads - 1) / threads;
    return b < 1 ? 1 : (b > 4096 ? 4096 : b);
  }

}  // namespace

// No C++ exception crosses the C ABI (see lst_event.cu): host-side failures
// become a -1 status with a message.
#define LST_ABI_TRY try {
#define LST_ABI_CATCH_INT        \
  }                              \
  catch (...) {                  \
    try {                        \
      g_dnnError = "host error"; \
    } catch (...) {              \
    }                            \
    return -1;                   \
  }

extern "C" {

size_t lst_t5dnn_scratch_floats(int n) {
  const size_t chunks = (size_t(n > 0 ? n : 0) + kChunk - 1) / kChunk;
  return 2 * size_t(kH) * size_t(n > 0 ? n : 0) + chunks * kParams;
}

int lst_t5dnn_forward(const float* weights, const float* x, int n, float* h1, float* h2, float* logit, void* stream) {
  LST_ABI_TRY
  if (n <= 0)
    return 0;
  if (!weights || !x || !h1 || !h2 || !logit)
    return -1;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaGetLastError();
  kDnnForward<<<blocksFor(n, 128), 128, 0, s>>>(weights, x, n, h1, h2, logit);
  if (cudaPeekAtLastError() != cudaSuccess)
    return dnnFail("kDnnForward");
  return 0;
  LST_ABI_CATCH_INT
}

int lst_t5dnn_backward(const float* weights, const float* x, const float* h1, const float* h2, const float* dlogit,
                       int n, float* grad, float* scratch, void* stream) {
  LST_ABI_TRY
  if (!weights || !x || !h1 || !h2 || !dlogit || !grad || !scratch)
    return -1;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaGetLastError();
  if (n <= 0) {
    if (cudaMemsetAsync(grad, 0, sizeof(float) * kParams, s) != cudaSuccess)
      return dnnFail("cudaMemsetAsync");
    return 0;
  }
  float* dh1 = scratch;
  float* dh2 = scratch + size_t(kH) * n;
  float* partial = scratch + 2 * size_t(kH) * n;
  const int nChunks = (n + kChunk - 1) / kChunk;
  kDnnBackSample<<<blocksFor(n, 128), 128, 0, s>>>(weights, h1, h2, dlogit, n, dh1, dh2);
  if (cudaPeekAtLastError() != cudaSuccess)
    return dnnFail("kDnnBackSample");
  kDnnGradPartial<<<dim3((kParams + 127) / 128, nChunks), 128, 0, s>>>(x, h1, h2, dlogit, dh1, dh2, n, partial);
  if (cudaPeekAtLastError() != cudaSuccess)
    return dnnFail("kDnnGradPartial");
  kDnnGradReduce<<<(kParams + 127) / 128, 128, 0, s>>>(partial, nChunks, grad);
  if (cudaPeekAtLastError() != cudaSuccess)
    return dnnFail("kDnnGradReduce");
  return 0;
  LST_ABI_CATCH_INT
}

const char* lst_t5dnn_last_error(void) { return g_dnnError.c_str(); }

}  // extern "C"
