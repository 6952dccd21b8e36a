// The format selector's network: MLP 12 -> 64 -> 64 -> 28 in FP32, ReLU on
// the hidden layers, trained with a masked mean-squared error on the log
// times of the 28 (format, launch configuration) pairs.
//
// Parameters are one flat FP32 array:
//   W1[12][64] b1[64] W2[64][64] b2[64] W3[64][28] b3[28]   (6,812 floats)
// (W[k][n] row-major: input k, output n).  Activations are row-major
// [batch][width].  Every kernel sums in a fixed order (no atomics), so a
// training run is reproducible bit for bit.
//
// The layers are a few thousand multiply-adds per sample, so the kernels are
// plain FP32 FMA loops: one thread per output element, the weight matrix of
// the layer staged in shared memory.
#pragma once

#include <cstdint>

namespace mfp {
namespace dev {

constexpr uint32_t kMlpIn = 12, kMlpHid = 64, kMlpOut = 28;
constexpr uint32_t kMlpW1 = 0, kMlpB1 = kMlpW1 + kMlpIn * kMlpHid, kMlpW2 = kMlpB1 + kMlpHid,
                   kMlpB2 = kMlpW2 + kMlpHid * kMlpHid, kMlpW3 = kMlpB2 + kMlpHid,
                   kMlpB3 = kMlpW3 + kMlpHid * kMlpOut, kMlpParams = kMlpB3 + kMlpOut;

// out[b][n] = act(sum_k in[b][k] * W[k][n] + bias[n]), K <= 64, N <= 64.
template <bool RELU>
__global__ void __launch_bounds__(256) mlp_dense_fwd(const float *__restrict__ in, const float *__restrict__ W,
                                                     const float *__restrict__ bias, float *__restrict__ out,
                                                     uint32_t B, uint32_t K, uint32_t N) {
  __shared__ float sW[64 * 64];
  __shared__ float sb[64];
  for (uint32_t i = threadIdx.x; i < K * N; i += blockDim.x) sW[i] = W[i];
  for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) sb[i] = bias[i];
  __syncthreads();
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (uint64_t)B * N) return;
  const uint32_t b = (uint32_t)(idx / N), n = (uint32_t)(idx % N);
  const float *x = in + (size_t)b * K;
  float acc = sb[n];
  for (uint32_t k = 0; k < K; ++k) acc = __fmaf_rn(x[k], sW[k * N + n], acc);
  out[idx] = RELU ? fmaxf(acc, 0.f) : acc;
}

// One CTA: loss = sum M (Y - T)^2 / sum M and dY = 2 M (Y - T) / sum M, in a
// fixed order (strided partial sums, then a tree over the CTA).
__global__ void __launch_bounds__(1024) mlp_loss_grad(const float *__restrict__ Y, const float *__restrict__ T,
                                                      const float *__restrict__ M, uint32_t n,
                                                      float *__restrict__ dY, float *__restrict__ loss) {
  __shared__ float s_m[1024], s_l[1024];
  float m = 0.f, l = 0.f;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    const float d = Y[i] - T[i];
    m += M[i];
    l = __fmaf_rn(M[i] * d, d, l);
  }
  s_m[threadIdx.x] = m;
  s_l[threadIdx.x] = l;
  __syncthreads();
  for (uint32_t h = blockDim.x / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      s_m[threadIdx.x] += s_m[threadIdx.x + h];
      s_l[threadIdx.x] += s_l[threadIdx.x + h];
    }
    __syncthreads();
  }
  const float inv = s_m[0] > 0.f ? 1.f / s_m[0] : 0.f;
  if (threadIdx.x == 0) *loss = s_l[0] * inv;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) dY[i] = 2.f * M[i] * (Y[i] - T[i]) * inv;
}

// dIn[b][k] = (sum_n dOut[b][n] * W[k][n]) * (H[b][k] > 0), the ReLU mask from
// the layer's input activations H (= dIn's forward values).
__global__ void __launch_bounds__(256) mlp_dense_bwd_in(const float *__restrict__ dOut, const float *__restrict__ W,
                                                        const float *__restrict__ H, float *__restrict__ dIn,
                                                        uint32_t B, uint32_t K, uint32_t N) {
  __shared__ float sW[64 * 64];
  for (uint32_t i = threadIdx.x; i < K * N; i += blockDim.x) sW[i] = W[i];
  __syncthreads();
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (uint64_t)B * K) return;
  const uint32_t b = (uint32_t)(idx / K), k = (uint32_t)(idx % K);
  const float *g = dOut + (size_t)b * N;
  float acc = 0.f;
  for (uint32_t n = 0; n < N; ++n) acc = __fmaf_rn(g[n], sW[k * N + n], acc);
  dIn[idx] = H[idx] > 0.f ? acc : 0.f;
}

// dW[k][n] = sum_b In[b][k] * dOut[b][n] (threads k*N + n < K*N) and
// db[n] = sum_b dOut[b][n] (threads K*N + n), b in increasing order.
__global__ void __launch_bounds__(256) mlp_dense_bwd_w(const float *__restrict__ in, const float *__restrict__ dOut,
                                                       float *__restrict__ dW, float *__restrict__ db, uint32_t B,
                                                       uint32_t K, uint32_t N) {
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < K * N) {
    const uint32_t k = idx / N, n = idx % N;
    float acc = 0.f;
    for (uint32_t b = 0; b < B; ++b) acc = __fmaf_rn(in[(size_t)b * K + k], dOut[(size_t)b * N + n], acc);
    dW[idx] = acc;
  } else if (idx < K * N + N) {
    const uint32_t n = idx - K * N;
    float acc = 0.f;
    for (uint32_t b = 0; b < B; ++b) acc += dOut[(size_t)b * N + n];
    db[n] = acc;
  }
}

// Adam (Kingma & Ba, 2015) with bias correction; step >= 1.
__global__ void __launch_bounds__(256) mlp_adam(float *__restrict__ p, const float *__restrict__ g,
                                                float *__restrict__ m, float *__restrict__ v, uint32_t n, float lr,
                                                float beta1, float beta2, float eps, float c1, float c2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = beta1 * m[i] + (1.f - beta1) * gi;
  const float vi = beta2 * v[i] + (1.f - beta2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace dev
}  // namespace mfp
