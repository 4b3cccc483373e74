// Entry points of the native runtime library libtfb200_runtime.so (built from
// tensorforge_b200/csrc/*.cu). None of them has a counterpart in the reference, which has
// no autotuner, records no rooflines and takes device buffers only: they back the learned
// cost model of the autotuner, the measured roofline denominators and the transfers of
// host-resident batches.
//
// Every function is asynchronous on `stream` (a cudaStream_t; nullptr = legacy default
// stream), allocates nothing, and returns the cudaError_t of its launch (0 = success).
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

// ---- throughput probes (roofline denominators)
// 16 independent FMA chains per thread, 256 threads per block, `iters` iterations;
// flops = 2 * 16 * iters * blocks * 256. `out` holds `blocks` values of the probe's type.
int tfb_fma_peak_launch(int is_double, void *out, int iters, int blocks, void *stream);
// 8 independent m8n8k4 FP64 MMA chains per warp, 8 warps per block, `iters` iterations;
// flops = 512 * 8 * iters * blocks * 8. `out` holds `blocks` doubles.
int tfb_dmma_peak_launch(void *out, int iters, int blocks, void *stream);
// tcgen05 TF32 MMAs of 128 x n x 8 (n = 16..256, multiple of 16) back to back into one
// accumulator, one CTA of 128 threads per block, A from tensor memory (a_smem = 0) or shared
// memory (1), B from shared memory; 1 + 8 * floor((iters - 1) / 8) MMAs per CTA, so flops =
// 2 * 128 * n * 8 * iters * blocks for iters = 8 k + 1. `err` (one device word) is raised to
// 1 if a CTA's bounded wait for its MMAs runs out.
int tfb_tc_tf32_peak_launch(int n, int a_smem, unsigned *err, int iters, int blocks, void *stream);

// ---- cost-model MLP, 32 -> 64 -> 64 -> 1 with ReLU, FP32
// Parameter vector (tfb_mlp_num_params() floats): W1[64][32], b1[64], W2[64][64], b2[64],
// W3[64], b3. Batches are row-major X[B][32]; T[B] are targets (log runtime).
int tfb_mlp_num_params(void);
// Y[B] = MLP(X); H1, H2 ([B][64] each) receive the hidden activations unless nullptr.
int tfb_mlp_forward(const float *params, const float *X, int B, float *H1, float *H2, float *Y, void *stream);
// Gradient of L = 1/(2B) sum (Y - T)^2 into grads (overwritten), from the activations of
// tfb_mlp_forward; dH1, dH2 ([B][64]) and dY ([B]) are scratch.
int tfb_mlp_backward(const float *params, const float *X, const float *T, int B, const float *H1,
                     const float *H2, const float *Y, float *dH1, float *dH2, float *dY, float *grads,
                     void *stream);
// out[0] = 1/(2B) sum (Y - T)^2
int tfb_mlp_loss(const float *Y, const float *T, int B, float *out, void *stream);
// One Adam step (bias-corrected with `step` >= 1) on n parameters; m, v are the moments.
int tfb_mlp_adam(float *params, const float *grads, float *m, float *v, int n, float lr, float b1, float b2,
                 float eps, int step, void *stream);

// ---- host-resident batches
// 2D copy: `rows` rows of `row_bytes` bytes, consecutive rows `src_pitch` / `dst_pitch` bytes
// apart; host -> device when to_device != 0, else device -> host. Host memory should be
// pinned for the copy to be asynchronous. Returns cudaErrorInvalidValue when a row is wider
// than a pitch.
int tfb_copy_rows_async(void *dst, size_t dst_pitch, const void *src, size_t src_pitch, size_t row_bytes,
                        size_t rows, int to_device, void *stream);

#ifdef __cplusplus
}
#endif
