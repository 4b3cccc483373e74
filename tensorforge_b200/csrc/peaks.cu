// CUDA-core FMA throughput probes: the denominators of the CUDA-core rooflines.
// No counterpart in the reference (which records no rooflines).
//
// Each thread runs 16 independent FMA chains for `iters` iterations, so the pipe is
// never latency bound; flops per launch = 2 * 16 * iters * blocks * threads.
#include <cuda_runtime.h>

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
