// The subdivision-level network of the adaptive IPM: 8 -> 64 -> 64 -> 5,
// ReLU hidden layers, softmax over the levels 1, 2, 4, 8, 16.
//
// Weights are held as FP32 masters and used as BF16 (round to nearest even)
// in the forward and backward passes; every product is accumulated in FP32.
// Inputs are standardised with the feature means and deviations stored with
// the network. Training minimises the mean cross-entropy of a minibatch with
// Adam; the passes are separate kernels:
//   mlp_train_forward   one thread per sample: activations, softmax, dL/dz3
//   mlp_train_backward  one thread per sample: dL/dz2, dL/dz1
//   mlp_grad            one thread per parameter: the minibatch sum, in sample
//                       order (deterministic)
//   mlp_adam            one thread per parameter: Adam step, BF16 copy
// Inference (mlp_classify) keeps the BF16 weights in shared memory as FP32
// and gives each thread one tile.
#pragma once
#include <cuda_bf16.h>

#include "common.cuh"

namespace irsb {

constexpr int kMlpIn = 8, kMlpH = 64, kMlpOut = 5;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kMlpH * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpH;
constexpr int kOffB2 = kOffW2 + kMlpH * kMlpH;
constexpr int kOffW3 = kOffB2 + kMlpH;
constexpr int kOffB3 = kOffW3 + kMlpOut * kMlpH;
constexpr int kMlpParams = kOffB3 + kMlpOut;  // 5061

__device__ __forceinline__ void mlp_stage(const __nv_bfloat16* __restrict__ w, float* sw) {
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) sw[i] = __bfloat162float(w[i]);
  __syncthreads();
}

__device__ __forceinline__ void mlp_inputs(const float* __restrict__ f, const float* __restrict__ mu,
                                           const float* __restrict__ sig, float* x) {
#pragma unroll
  for (int i = 0; i < kMlpIn; i++) x[i] = (f[i] - mu[i]) / sig[i];
}

// Logits of one sample; h1 / h2 (if given) receive the hidden activations.
__device__ __forceinline__ void mlp_logits(const float* sw, const float* x, float* h1, float* h2, float* z3) {
#pragma unroll
  for (int o = 0; o < kMlpH; o++) {
    float a = sw[kOffB1 + o];
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) a = fmaf(sw[kOffW1 + o * kMlpIn + i], x[i], a);
    h1[o] = a > 0.f ? a : 0.f;
  }
#pragma unroll
  for (int k = 0; k < kMlpOut; k++) z3[k] = sw[kOffB3 + k];
  for (int o = 0; o < kMlpH; o++) {
    float a = sw[kOffB2 + o];
#pragma unroll 16
    for (int i = 0; i < kMlpH; i++) a = fmaf(sw[kOffW2 + o * kMlpH + i], h1[i], a);
    a = a > 0.f ? a : 0.f;
    if (h2) h2[o] = a;
#pragma unroll
    for (int k = 0; k < kMlpOut; k++) z3[k] = fmaf(sw[kOffW3 + k * kMlpH + o], a, z3[k]);
  }
}

// Level class of each sample: the argmax of the logits (q <= 0), or the
// smallest class whose cumulative softmax probability reaches q (the classes
// are ordered levels; q > 0.5 leans towards refining).
__global__ void __launch_bounds__(128) mlp_classify(const __nv_bfloat16* __restrict__ w, const float* __restrict__ mu,
                                                    const float* __restrict__ sig, const float* __restrict__ feat,
                                                    int n, float q, int* __restrict__ cls) {
  __shared__ float sw[kMlpParams];
  mlp_stage(w, sw);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    float x[kMlpIn], h1[kMlpH], z3[kMlpOut];
    mlp_inputs(feat + (long long)s * kMlpIn, mu, sig, x);
    mlp_logits(sw, x, h1, nullptr, z3);
    int best = 0;
#pragma unroll
    for (int k = 1; k < kMlpOut; k++)
      if (z3[k] > z3[best]) best = k;
    if (q > 0.f) {
      float e[kMlpOut], se = 0.f;
#pragma unroll
      for (int k = 0; k < kMlpOut; k++) {
        e[k] = expf(z3[k] - z3[best]);
        se += e[k];
      }
      float cum = 0.f;
      best = kMlpOut - 1;
      for (int k = 0; k < kMlpOut; k++) {
        cum += e[k] / se;
        if (cum >= q) {
          best = k;
          break;
        }
      }
    }
    cls[s] = best;
  }
}

// Minibatch of B samples idx[0..B): activations, per-sample loss and
// d(mean loss)/d z3.
__global__ void __launch_bounds__(128) mlp_train_forward(const __nv_bfloat16* __restrict__ w,
                                                         const float* __restrict__ mu, const float* __restrict__ sig,
                                                         const float* __restrict__ feat, const int* __restrict__ label,
                                                         const int* __restrict__ idx, int B, float* __restrict__ X,
                                                         float* __restrict__ H1, float* __restrict__ H2,
                                                         float* __restrict__ D3, float* __restrict__ loss) {
  __shared__ float sw[kMlpParams];
  mlp_stage(w, sw);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < B; s += gridDim.x * blockDim.x) {
    const int n = idx[s];
    float x[kMlpIn], h1[kMlpH], h2[kMlpH], z3[kMlpOut];
    mlp_inputs(feat + (long long)n * kMlpIn, mu, sig, x);
    mlp_logits(sw, x, h1, h2, z3);
    float m = z3[0];
#pragma unroll
    for (int k = 1; k < kMlpOut; k++) m = fmaxf(m, z3[k]);
    float e[kMlpOut], se = 0.f;
#pragma unroll
    for (int k = 0; k < kMlpOut; k++) {
      e[k] = expf(z3[k] - m);
      se += e[k];
    }
    const int y = label[n];
    loss[s] = logf(se) - (z3[y] - m);
#pragma unroll
    for (int k = 0; k < kMlpOut; k++) D3[s * kMlpOut + k] = (e[k] / se - (k == y ? 1.f : 0.f)) / float(B);
#pragma unroll
    for (int i = 0; i < kMlpIn; i++) X[s * kMlpIn + i] = x[i];
    for (int o = 0; o < kMlpH; o++) {
      H1[s * kMlpH + o] = h1[o];
      H2[s * kMlpH + o] = h2[o];
    }
  }
}

__global__ void __launch_bounds__(128) mlp_train_backward(const __nv_bfloat16* __restrict__ w, int B,
                                                          const float* __restrict__ H1, const float* __restrict__ H2,
                                                          const float* __restrict__ D3, float* __restrict__ D2,
                                                          float* __restrict__ D1) {
  __shared__ float sw[kMlpParams];
  mlp_stage(w, sw);
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < B; s += gridDim.x * blockDim.x) {
    float d3[kMlpOut], d2[kMlpH];
#pragma unroll
    for (int k = 0; k < kMlpOut; k++) d3[k] = D3[s * kMlpOut + k];
    for (int o = 0; o < kMlpH; o++) {
      float a = 0.f;
#pragma unroll
      for (int k = 0; k < kMlpOut; k++) a = fmaf(sw[kOffW3 + k * kMlpH + o], d3[k], a);
      d2[o] = H2[s * kMlpH + o] > 0.f ? a : 0.f;
      D2[s * kMlpH + o] = d2[o];
    }
    for (int i = 0; i < kMlpH; i++) {
      float a = 0.f;
#pragma unroll 16
      for (int o = 0; o < kMlpH; o++) a = fmaf(sw[kOffW2 + o * kMlpH + i], d2[o], a);
      D1[s * kMlpH + i] = H1[s * kMlpH + i] > 0.f ? a : 0.f;
    }
  }
}

// Gradient of the mean loss for every parameter, summed over the minibatch in
// sample order.
__global__ void mlp_grad(int B, const float* __restrict__ X, const float* __restrict__ H1,
                         const float* __restrict__ H2, const float* __restrict__ D1, const float* __restrict__ D2,
                         const float* __restrict__ D3, float* __restrict__ grad) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < kMlpParams; q += gridDim.x * blockDim.x) {
    const float* d;
    const float* a = nullptr;
    int dn, an = 0, o, i = 0;
    if (q < kOffB1) {
      o = (q - kOffW1) / kMlpIn, i = (q - kOffW1) % kMlpIn, d = D1, dn = kMlpH, a = X, an = kMlpIn;
    } else if (q < kOffW2) {
      o = q - kOffB1, d = D1, dn = kMlpH;
    } else if (q < kOffB2) {
      o = (q - kOffW2) / kMlpH, i = (q - kOffW2) % kMlpH, d = D2, dn = kMlpH, a = H1, an = kMlpH;
    } else if (q < kOffW3) {
      o = q - kOffB2, d = D2, dn = kMlpH;
    } else if (q < kOffB3) {
      o = (q - kOffW3) / kMlpH, i = (q - kOffW3) % kMlpH, d = D3, dn = kMlpOut, a = H2, an = kMlpH;
    } else {
      o = q - kOffB3, d = D3, dn = kMlpOut;
    }
    float g = 0.f;
    for (int s = 0; s < B; s++) g = fmaf(d[s * dn + o], a ? a[s * an + i] : 1.f, g);
    grad[q] = g;
  }
}

__global__ void mlp_adam(int step, float lr, float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                         const float* __restrict__ grad, __nv_bfloat16* __restrict__ wb) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < kMlpParams; q += gridDim.x * blockDim.x) {
    const float g = grad[q];
    const float mq = b1 * m[q] + (1.f - b1) * g;
    const float vq = b2 * v[q] + (1.f - b2) * g * g;
    m[q] = mq;
    v[q] = vq;
    const float wq = w[q] - lr * (mq / c1) / (sqrtf(vq / c2) + eps);
    w[q] = wq;
    wb[q] = __float2bfloat16_rn(wq);
  }
}

__global__ void mlp_to_bf16(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < kMlpParams; q += gridDim.x * blockDim.x)
    wb[q] = __float2bfloat16_rn(w[q]);
}

}  // namespace irsb
