// Throughput probes: the denominators of the CUDA-core and FP64 tensor-core rooflines.
// No counterpart in the reference (which records no rooflines).
//
// FMA probe: each thread runs 16 independent FMA chains for `iters` iterations, so the
// pipe is never latency bound; flops per launch = 2 * 16 * iters * blocks * threads.
// DMMA probe: each warp runs 8 independent m8n8k4 FP64 MMA chains; flops per launch =
// 512 * 8 * iters * blocks * warps.
#include <cuda_runtime.h>
#include "tensorforge_b200_runtime.h"

template <typename T>
__global__ void __launch_bounds__(256) fma_peak_kernel(T *out, int iters, T seed) {
  T a[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) a[i] = seed + (T)(threadIdx.x + i);
  const T b = (T)0.999999, c = (T)1e-7;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = a[i] * b + c;
  }
  T s = 0;
#pragma unroll
  for (int i = 0; i < 16; ++i) s += a[i];
  if (s == (T)-1.2345) out[blockIdx.x] = s;  // keeps the chains live
}

extern "C" int tfb_fma_peak_launch(int is_double, void *out, int iters, int blocks, void *stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (is_double) {
    fma_peak_kernel<double><<<blocks, 256, 0, st>>>(static_cast<double *>(out), iters, 1.0);
  } else {
    fma_peak_kernel<float><<<blocks, 256, 0, st>>>(static_cast<float *>(out), iters, 1.0f);
  }
  return static_cast<int>(cudaGetLastError());
}

__global__ void __launch_bounds__(256) dmma_peak_kernel(double *out, int iters) {
  const unsigned lane = threadIdx.x & 31u;
  double d[8][2];
#pragma unroll
  for (int i = 0; i < 8; ++i) { d[i][0] = 0.0; d[i][1] = 0.0; }
  const double a = 1e-3 * (double)(lane + 1), b = 1e-3 * (double)(33 - lane);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                   : "+d"(d[i][0]), "+d"(d[i][1]) : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += d[i][0] + d[i][1];
  if (s == -1.2345) out[blockIdx.x] = s;  // keeps the chains live
}

extern "C" int tfb_dmma_peak_launch(void *out, int iters, int blocks, void *stream) {
  dmma_peak_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<double *>(out), iters);
  return static_cast<int>(cudaGetLastError());
}
