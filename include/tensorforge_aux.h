// Runtime helpers used by every generated launcher.
//
// Replaces tensorforge/include/tensorforge_aux.h:1-15 (CHECK_ERR, tensorforge::checkErr,
// tensorforge::synchDevice) with the same names and meaning, for the CUDA backend on
// B200. Differences: checkErr never throws (each launcher is also called from its C-linkage
// twin tfb_launch_<name>, which must not unwind into C or ctypes callers); it records the CUDA error as a status code, readable and clearable through
// tensorforge_last_status(), and prints it unless NDEBUG is defined.
#ifndef TENSORFORGE_INTERNALS_H
#define TENSORFORGE_INTERNALS_H

#ifdef __cplusplus
#include <string>

#define CHECK_ERR tensorforge::checkErr(__FILE__, __LINE__)

namespace tensorforge {
  void checkErr(const std::string &file, int line);
  void synchDevice(void *stream = nullptr);
}  // namespace tensorforge

extern "C" {
#endif

// Last CUDA error recorded by CHECK_ERR in the calling thread (0 = none); clears it.
// No counterpart in the reference, whose checkErr throws instead.
int tensorforge_last_status(void);

// Status-returning form of tensorforge::synchDevice (cudaStreamSynchronize on the given
// stream, or cudaDeviceSynchronize for nullptr); returns the CUDA error code.
int tensorforge_synch_device(void *stream);

#ifdef __cplusplus
}
#endif

#endif  // TENSORFORGE_INTERNALS_H
