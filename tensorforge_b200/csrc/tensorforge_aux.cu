// Implementation of include/tensorforge_aux.h (see there). Replaces
// tensorforge/include/tensorforge_aux.cu:1-37.
#include <cstdio>
#include <string>
#include <cuda_runtime.h>
#include "tensorforge_aux.h"

namespace {
thread_local int tfb_last_status = 0;
// a copy: the caller's string is usually a temporary built from __FILE__
thread_local std::string tfb_prev_file;
thread_local int tfb_prev_line = 0;
}  // namespace

namespace tensorforge {

void checkErr(const std::string &file, int line) {
  cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    tfb_last_status = static_cast<int>(err);
#ifndef NDEBUG
    std::fprintf(stderr, "\n%s, line %d: %s (%d)\n", file.c_str(), line, cudaGetErrorString(err),
                 static_cast<int>(err));
    if (tfb_prev_line > 0) std::fprintf(stderr, "Previous CUDA call:\n%s, line %d\n", tfb_prev_file.c_str(), tfb_prev_line);
#endif
    return;
  }
  tfb_prev_file = file;
  tfb_prev_line = line;
}

void synchDevice(void *stream) {
  if (stream != nullptr) {
    cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  } else {
    cudaDeviceSynchronize();
  }
  checkErr(__FILE__, __LINE__);
}

}  // namespace tensorforge

extern "C" int tensorforge_last_status(void) {
  int s = tfb_last_status;
  tfb_last_status = 0;
  return s;
}

extern "C" int tensorforge_synch_device(void *stream) {
  cudaError_t err = (stream != nullptr) ? cudaStreamSynchronize(static_cast<cudaStream_t>(stream))
                                        : cudaDeviceSynchronize();
  return static_cast<int>(err);
}
