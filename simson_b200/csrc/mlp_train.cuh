// Training of the learned SGS model (no counterpart in the reference): full-
// batch Adam on the mean squared error of
//   y = W3 tanh(W2 tanh(W1 x + b1) + b2) + b3,   L = sum (y - t)^2 / (6 n),
// x the ten features and t the six target stresses of n samples (scaled as
// the caller wants them at inference: sgpu_sgs_mlp's s_in, s_y, s_out).
// FP32 master weights, packed: W1 [64][10], b1 [64], W2 [64][64], b2 [64],
// W3 [6][64], b3 [6] (5254 values, the layout of sgpu_sgs_mlp).
//
//   k_mlp_grad    one CTA per chunk of MLP_CHUNK samples: forward pass,
//                 backward pass, the chunk's partial gradient of every
//                 weight and its partial loss (weights and activations in
//                 shared memory, FP32)
//   k_mlp_reduce  per weight: the chunks' partials summed in chunk order
//   k_mlp_adam    per weight: Adam (beta1 0.9, beta2 0.999, eps 1e-8) with
//                 the bias corrections passed by the host
#pragma once
#include <cuda_runtime.h>

namespace sb {

constexpr int MLP_NIN = 10, MLP_NH = 64, MLP_NOUT = 6;
constexpr int MLP_OW1 = 0, MLP_OB1 = 640, MLP_OW2 = 704, MLP_OB2 = 4800, MLP_OW3 = 4864, MLP_OB3 = 5248;
constexpr int MLP_NPAR = 5254;
constexpr int MLP_CHUNK = 64;
constexpr int MLP_TRAIN_THREADS = 256;
// shared memory of k_mlp_grad: weights, x, h1, h2, dy, g2, g1, loss partials
constexpr size_t MLP_TRAIN_SMEM =
    sizeof(float) * (MLP_NPAR + MLP_CHUNK * (MLP_NIN + 4 * MLP_NH + MLP_NOUT) + MLP_TRAIN_THREADS);

// part: [nchunk][MLP_NPAR + 1] (the last entry the chunk's sum of squared errors)
__global__ void __launch_bounds__(MLP_TRAIN_THREADS) k_mlp_grad(const float* __restrict__ par,
                                                              const float* __restrict__ x,
                                                              const float* __restrict__ t, long long n,
                                                              float* __restrict__ part) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float* P = reinterpret_cast<float*>(smem_raw);
  float* X = P + MLP_NPAR;
  float* H1 = X + MLP_CHUNK * MLP_NIN;
  float* H2 = H1 + MLP_CHUNK * MLP_NH;
  float* G2 = H2 + MLP_CHUNK * MLP_NH;
  float* G1 = G2 + MLP_CHUNK * MLP_NH;
  float* D3 = G1 + MLP_CHUNK * MLP_NH;
  float* red = D3 + MLP_CHUNK * MLP_NOUT;
  const int tid = threadIdx.x;
  const long long s0 = (long long)blockIdx.x * MLP_CHUNK;
  const float inv = 2.0f / (6.0f * (float)n);
  for (int e = tid; e < MLP_NPAR; e += MLP_TRAIN_THREADS) P[e] = par[e];
  for (int e = tid; e < MLP_CHUNK * MLP_NIN; e += MLP_TRAIN_THREADS) {
    const long long s = s0 + e / MLP_NIN;
    X[e] = (s < n) ? x[s0 * MLP_NIN + e] : 0.0f;
  }
  __syncthreads();
  for (int e = tid; e < MLP_CHUNK * MLP_NH; e += MLP_TRAIN_THREADS) {
    const int s = e / MLP_NH, j = e - s * MLP_NH;
    float a = P[MLP_OB1 + j];
    for (int k = 0; k < MLP_NIN; ++k) a = fmaf(P[MLP_OW1 + j * MLP_NIN + k], X[s * MLP_NIN + k], a);
    H1[e] = tanhf(a);
  }
  __syncthreads();
  for (int e = tid; e < MLP_CHUNK * MLP_NH; e += MLP_TRAIN_THREADS) {
    const int s = e / MLP_NH, j = e - s * MLP_NH;
    float a = P[MLP_OB2 + j];
    for (int k = 0; k < MLP_NH; ++k) a = fmaf(P[MLP_OW2 + j * MLP_NH + k], H1[s * MLP_NH + k], a);
    H2[e] = tanhf(a);
  }
  __syncthreads();
  float sq = 0.0f;
  for (int e = tid; e < MLP_CHUNK * MLP_NOUT; e += MLP_TRAIN_THREADS) {
    const int s = e / MLP_NOUT, o = e - s * MLP_NOUT;
    float d = 0.0f;
    if (s0 + s < n) {
      float y = P[MLP_OB3 + o];
      for (int k = 0; k < MLP_NH; ++k) y = fmaf(P[MLP_OW3 + o * MLP_NH + k], H2[s * MLP_NH + k], y);
      const float r = y - t[s0 * MLP_NOUT + e];
      sq = fmaf(r, r, sq);
      d = inv * r;
    }
    D3[e] = d;
  }
  red[tid] = sq;
  __syncthreads();
  for (int e = tid; e < MLP_CHUNK * MLP_NH; e += MLP_TRAIN_THREADS) {
    const int s = e / MLP_NH, j = e - s * MLP_NH;
    float g = 0.0f;
    for (int o = 0; o < MLP_NOUT; ++o) g = fmaf(D3[s * MLP_NOUT + o], P[MLP_OW3 + o * MLP_NH + j], g);
    const float h = H2[e];
    G2[e] = g * (1.0f - h * h);
  }
  __syncthreads();
  for (int e = tid; e < MLP_CHUNK * MLP_NH; e += MLP_TRAIN_THREADS) {
    const int s = e / MLP_NH, j = e - s * MLP_NH;
    float g = 0.0f;
    for (int i = 0; i < MLP_NH; ++i) g = fmaf(G2[s * MLP_NH + i], P[MLP_OW2 + i * MLP_NH + j], g);
    const float h = H1[e];
    G1[e] = g * (1.0f - h * h);
  }
  __syncthreads();
  float* out = part + (size_t)blockIdx.x * (MLP_NPAR + 1);
  for (int e = tid; e < MLP_NPAR; e += MLP_TRAIN_THREADS) {
    float g = 0.0f;
    if (e < MLP_OB1) {
      const int j = e / MLP_NIN, k = e - j * MLP_NIN;
      for (int s = 0; s < MLP_CHUNK; ++s) g = fmaf(G1[s * MLP_NH + j], X[s * MLP_NIN + k], g);
    } else if (e < MLP_OW2) {
      const int j = e - MLP_OB1;
      for (int s = 0; s < MLP_CHUNK; ++s) g += G1[s * MLP_NH + j];
    } else if (e < MLP_OB2) {
      const int j = (e - MLP_OW2) / MLP_NH, k = (e - MLP_OW2) - j * MLP_NH;
      for (int s = 0; s < MLP_CHUNK; ++s) g = fmaf(G2[s * MLP_NH + j], H1[s * MLP_NH + k], g);
    } else if (e < MLP_OW3) {
      const int j = e - MLP_OB2;
      for (int s = 0; s < MLP_CHUNK; ++s) g += G2[s * MLP_NH + j];
    } else if (e < MLP_OB3) {
      const int o = (e - MLP_OW3) / MLP_NH, k = (e - MLP_OW3) - o * MLP_NH;
      for (int s = 0; s < MLP_CHUNK; ++s) g = fmaf(D3[s * MLP_NOUT + o], H2[s * MLP_NH + k], g);
    } else {
      const int o = e - MLP_OB3;
      for (int s = 0; s < MLP_CHUNK; ++s) g += D3[s * MLP_NOUT + o];
    }
    out[e] = g;
  }
  if (tid == 0) {
    float l = 0.0f;
    for (int i = 0; i < MLP_TRAIN_THREADS; ++i) l += red[i];
    out[MLP_NPAR] = l;
  }
}

// grad[e] = sum over chunks, in chunk order (grad[MLP_NPAR]: sum of squared errors)
__global__ void k_mlp_reduce(const float* __restrict__ part, int nchunk, float* __restrict__ grad) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e > MLP_NPAR) return;
  float g = 0.0f;
  for (int c = 0; c < nchunk; ++c) g += part[(size_t)c * (MLP_NPAR + 1) + e];
  grad[e] = g;
}

// c1 = 1 / (1 - beta1^step), c2 = 1 / (1 - beta2^step)
__global__ void k_mlp_adam(float* __restrict__ par, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ grad, float lr, float c1, float c2) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= MLP_NPAR) return;
  const float g = grad[e];
  const float mm = 0.9f * m[e] + 0.1f * g;
  const float vv = 0.999f * v[e] + 0.001f * g * g;
  m[e] = mm;
  v[e] = vv;
  par[e] = par[e] - lr * (mm * c1) / (sqrtf(vv * c2) + 1e-8f);
}

}  // namespace sb
