// Throughput probes: the denominators of the CUDA-core and FP64 tensor-core rooflines.
// No counterpart in the reference (which records no rooflines).
//
// FMA probe: each thread runs 16 independent FMA chains for `iters` iterations, so the
// pipe is never latency bound; flops per launch = 2 * 16 * iters * blocks * threads.
// DMMA probe: each warp runs 8 independent m8n8k4 FP64 MMA chains; flops per launch =
// 512 * 8 * iters * blocks * warps.
#include <cstdint>
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

// tcgen05 TF32 probe: one CTA per SM issues 1 + 8 * floor((iters - 1) / 8) MMAs of
// 128 x n x 8 (kind::tf32, one accumulator in tensor memory; A from tensor memory or, with
// a_smem, from shared memory; B from shared memory; operands zero) back to back, commits
// them to an mbarrier and waits for them; flops per launch = 2 * 128 * n * 8 * iters *
// blocks for iters = 8 k + 1. The wait is bounded: on timeout the
// CTA records error 1 in `err` and still releases its tensor memory.
namespace {
__device__ __forceinline__ unsigned tc_smem_u32(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ uint64_t tc_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFFu) >> 4);
  d |= (uint64_t)((lbo & 0x3FFFFu) >> 4) << 16;
  d |= (uint64_t)((sbo & 0x3FFFFu) >> 4) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
}  // namespace

__global__ void __launch_bounds__(128, 1) tc_tf32_peak_kernel(int iters, int n, int a_smem, unsigned* err) {
  // A: 128 rows x 8 K values, B: up to 256 rows x 8 K values (canonical K-major, no swizzle)
  __shared__ __align__(1024) float sa[128 * 8];
  __shared__ __align__(1024) float sb[256 * 8];
  __shared__ __align__(8) uint64_t bar;
  __shared__ unsigned tmem_slot;
  for (int i = threadIdx.x; i < 128 * 8; i += blockDim.x) sa[i] = 0.0f;
  for (int i = threadIdx.x; i < 256 * 8; i += blockDim.x) sb[i] = 0.0f;
  const unsigned warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(tc_smem_u32(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" :: "r"(tc_smem_u32(&tmem_slot)) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const unsigned tmem = tmem_slot;
  if (threadIdx.x == 0) {
    const unsigned idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(n >> 3) << 17) | ((128u >> 4) << 24);
    const uint64_t bd = tc_desc(tc_smem_u32(sb), 128u, 256u);
    const uint64_t ad = tc_desc(tc_smem_u32(sa), 128u, 256u);
    // one accumulation chain, as the K steps of a GEMM; the issue loop is unrolled by 8 so
    // that it does not bound the rate
    const unsigned d = tmem + 256u;
#define TFB_TC_PROBE_MMA(ACC)                                                                   \
    if (a_smem) {                                                                               \
      asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"                              \
                   " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}"               \
                   :: "r"(d), "l"(ad), "l"(bd), "r"(idesc), "r"(ACC) : "memory");              \
    } else {                                                                                    \
      asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"                              \
                   " tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}"             \
                   :: "r"(d), "r"(tmem), "l"(bd), "r"(idesc), "r"(ACC) : "memory");            \
    }
    TFB_TC_PROBE_MMA(0u)
    for (int it = 1; it + 8 <= iters; it += 8) {
      TFB_TC_PROBE_MMA(1u) TFB_TC_PROBE_MMA(1u) TFB_TC_PROBE_MMA(1u) TFB_TC_PROBE_MMA(1u)
      TFB_TC_PROBE_MMA(1u) TFB_TC_PROBE_MMA(1u) TFB_TC_PROBE_MMA(1u) TFB_TC_PROBE_MMA(1u)
    }
#undef TFB_TC_PROBE_MMA
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(tc_smem_u32(&bar)) : "memory");
    bool done = false;
    for (unsigned long long poll = 0; poll < (1ull << 26) && !done; ++poll) {
      unsigned ok;
      asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
                   : "=r"(ok) : "r"(tc_smem_u32(&bar)) : "memory");
      done = ok != 0;
    }
    if (!done) atomicMax(err, 1u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" :: "r"(tmem) : "memory");
  }
}

extern "C" int tfb_tc_tf32_peak_launch(int n, int a_smem, unsigned *err, int iters, int blocks, void *stream) {
  if (n < 16 || n > 256 || n % 16 != 0) return static_cast<int>(cudaErrorInvalidValue);
  tc_tf32_peak_kernel<<<blocks, 128, 0, static_cast<cudaStream_t>(stream)>>>(iters, n, a_smem, err);
  return static_cast<int>(cudaGetLastError());
}
