// Host <-> device transfers of per-element slots for batches that live in host memory.
// No counterpart in the reference, whose launchers only take device buffers.
//
// A compactly stored sparse operand occupies the first `row_bytes` of each element's slot
// (the slot is the tensor's full volume); the kernel reads only those, so a host-resident
// batch needs only them on the device: one 2D copy moves `rows` rows of `row_bytes` bytes
// between slots `pitch` bytes apart on both sides.
#include <cuda_runtime.h>
#include "tensorforge_b200_runtime.h"

extern "C" int tfb_copy_rows_async(void *dst, size_t dst_pitch, const void *src, size_t src_pitch,
                                   size_t row_bytes, size_t rows, int to_device, void *stream) {
  if (rows == 0 || row_bytes == 0) return 0;
  if (row_bytes > dst_pitch || row_bytes > src_pitch) return (int)cudaErrorInvalidValue;
  return (int)cudaMemcpy2DAsync(dst, dst_pitch, src, src_pitch, row_bytes, rows,
                                to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost,
                                static_cast<cudaStream_t>(stream));
}
