// MLP cost model kernels: 32 -> 64 -> 64 -> 1 (ReLU), FP32, trained with MSE on log-runtime.
// No counterpart in the reference (which has no autotuner).
//
// Parameter vector layout (TFB_MLP_PARAMS floats): W1[64][32], b1[64], W2[64][64], b2[64],
// W3[64], b3[1] (row-major, y = W x + b). Batches are row-major [B][features]. Scratch
// buffers (activations, per-sample deltas) are passed in by the caller.
#include <cuda_runtime.h>
#include "tensorforge_b200_runtime.h"

#define TFB_MLP_IN 32
#define TFB_MLP_H 64
#define TFB_MLP_PARAMS (TFB_MLP_H * TFB_MLP_IN + TFB_MLP_H + TFB_MLP_H * TFB_MLP_H + TFB_MLP_H + TFB_MLP_H + 1)

namespace {
constexpr int IN = TFB_MLP_IN, H = TFB_MLP_H;
constexpr int OW1 = 0, OB1 = OW1 + H * IN, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + H;

// one thread per sample: the weights are read by all threads in the same order (broadcast)
__global__ void mlp_forward_kernel(const float* __restrict__ p, const float* __restrict__ X, int B,
                                   float* __restrict__ H1, float* __restrict__ H2, float* __restrict__ Y) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  float x[IN];
#pragma unroll
  for (int i = 0; i < IN; ++i) x[i] = X[(size_t)b * IN + i];
  float h1[H];
#pragma unroll 4
  for (int u = 0; u < H; ++u) {
    float s = p[OB1 + u];
#pragma unroll
    for (int i = 0; i < IN; ++i) s = fmaf(p[OW1 + u * IN + i], x[i], s);
    h1[u] = s > 0.f ? s : 0.f;
    if (H1) H1[(size_t)b * H + u] = h1[u];
  }
  float y = p[OB3];
  for (int u = 0; u < H; ++u) {
    float s = p[OB2 + u];
#pragma unroll 8
    for (int i = 0; i < H; ++i) s = fmaf(p[OW2 + u * H + i], h1[i], s);
    const float h2 = s > 0.f ? s : 0.f;
    if (H2) H2[(size_t)b * H + u] = h2;
    y = fmaf(p[OW3 + u], h2, y);
  }
  Y[b] = y;
}

// per-sample deltas of L = 1/(2B) sum_b (y_b - t_b)^2
__global__ void mlp_backward_samples_kernel(const float* __restrict__ p, const float* __restrict__ T, int B,
                                            const float* __restrict__ H1, const float* __restrict__ H2,
                                            const float* __restrict__ Y, float* __restrict__ dH1,
                                            float* __restrict__ dH2, float* __restrict__ dY) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const float dy = (Y[b] - T[b]) / (float)B;
  dY[b] = dy;
  float d2[H];
  for (int u = 0; u < H; ++u) {
    const float h2 = H2[(size_t)b * H + u];
    d2[u] = h2 > 0.f ? dy * p[OW3 + u] : 0.f;
    dH2[(size_t)b * H + u] = d2[u];
  }
  for (int i = 0; i < H; ++i) {
    float s = 0.f;
    for (int u = 0; u < H; ++u) s = fmaf(p[OW2 + u * H + i], d2[u], s);
    const float h1 = H1[(size_t)b * H + i];
    dH1[(size_t)b * H + i] = h1 > 0.f ? s : 0.f;
  }
}

// one thread per parameter: reduce the per-sample outer products over the batch
__global__ void mlp_param_grads_kernel(const float* __restrict__ X, int B, const float* __restrict__ H1,
                                       const float* __restrict__ H2, const float* __restrict__ dH1,
                                       const float* __restrict__ dH2, const float* __restrict__ dY,
                                       float* __restrict__ g) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= TFB_MLP_PARAMS) return;
  float s = 0.f;
  if (q < OB1) {
    const int u = q / IN, i = q - u * IN;
    for (int b = 0; b < B; ++b) s = fmaf(dH1[(size_t)b * H + u], X[(size_t)b * IN + i], s);
  } else if (q < OW2) {
    const int u = q - OB1;
    for (int b = 0; b < B; ++b) s += dH1[(size_t)b * H + u];
  } else if (q < OB2) {
    const int r = q - OW2, u = r / H, i = r - u * H;
    for (int b = 0; b < B; ++b) s = fmaf(dH2[(size_t)b * H + u], H1[(size_t)b * H + i], s);
  } else if (q < OW3) {
    const int u = q - OB2;
    for (int b = 0; b < B; ++b) s += dH2[(size_t)b * H + u];
  } else if (q < OB3) {
    const int u = q - OW3;
    for (int b = 0; b < B; ++b) s = fmaf(dY[b], H2[(size_t)b * H + u], s);
  } else {
    for (int b = 0; b < B; ++b) s += dY[b];
  }
  g[q] = s;
}

__global__ void mlp_loss_kernel(const float* __restrict__ Y, const float* __restrict__ T, int B, float* __restrict__ out) {
  __shared__ float part[256];
  float s = 0.f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const float d = Y[b] - T[b];
    s = fmaf(d, d, s);
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = part[0] / (2.f * (float)B);
}

__global__ void mlp_adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                                float* __restrict__ v, int n, float lr, float b1, float b2, float eps,
                                float c1, float c2) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float gq = g[q];
  const float mq = b1 * m[q] + (1.f - b1) * gq;
  const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
  m[q] = mq;
  v[q] = vq;
  p[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
}
}  // namespace

extern "C" int tfb_mlp_num_params(void) { return TFB_MLP_PARAMS; }

extern "C" int tfb_mlp_forward(const float* params, const float* X, int B, float* H1, float* H2, float* Y,
                               void* stream) {
  if (B <= 0) return 0;
  mlp_forward_kernel<<<(B + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(params, X, B, H1, H2, Y);
  return static_cast<int>(cudaGetLastError());
}

extern "C" int tfb_mlp_backward(const float* params, const float* X, const float* T, int B, const float* H1,
                                const float* H2, const float* Y, float* dH1, float* dH2, float* dY,
                                float* grads, void* stream) {
  if (B <= 0) return 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  mlp_backward_samples_kernel<<<(B + 127) / 128, 128, 0, st>>>(params, T, B, H1, H2, Y, dH1, dH2, dY);
  mlp_param_grads_kernel<<<(TFB_MLP_PARAMS + 127) / 128, 128, 0, st>>>(X, B, H1, H2, dH1, dH2, dY, grads);
  return static_cast<int>(cudaGetLastError());
}

extern "C" int tfb_mlp_loss(const float* Y, const float* T, int B, float* out, void* stream) {
  if (B <= 0) return 0;
  mlp_loss_kernel<<<1, 256, 0, static_cast<cudaStream_t>(stream)>>>(Y, T, B, out);
  return static_cast<int>(cudaGetLastError());
}

extern "C" int tfb_mlp_adam(float* params, const float* grads, float* m, float* v, int n, float lr, float b1,
                            float b2, float eps, int step, void* stream) {
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  mlp_adam_kernel<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(params, grads, m, v, n, lr, b1,
                                                                                  b2, eps, c1, c2);
  return static_cast<int>(cudaGetLastError());
}
