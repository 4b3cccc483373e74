// Grouped (mixed-shape) launches generated by tensorforge_b200.grouped.GroupedKernel.
//
// A grouped library fuses several generated chains (the same operation at different basis
// sizes / quantity counts) into one persistent kernel. Its entry points carry the name of
// the fused set, `<set>`, and are declared with TFB_GROUPED_DECLARE(<set>). They have no
// counterpart in the reference, which launches one kernel per shape
// (tensorforge/generators/generator.py:164-196).
#ifndef TENSORFORGE_B200_GROUPED_H
#define TENSORFORGE_B200_GROUPED_H

#include <cuda_runtime.h>

#define TFB_GROUP_MAX_SYMBOLS 16

#ifndef TFB_GROUP_ARGS
#define TFB_GROUP_ARGS
// One group's launcher arguments: its ABI symbols in launcher order (pointer, or device
// array of pointers for pointer-addressed operands) with their extra offsets, the element
// count and the optional per-element flags (nullptr = all elements).
struct tfb_group_args {
  const void* ptr[TFB_GROUP_MAX_SYMBOLS];
  unsigned off[TFB_GROUP_MAX_SYMBOLS];
  unsigned long long num_elements;
  const unsigned* flags;
};
#endif

// Largest number of groups the allocation-free entry point accepts (its group records
// travel as one kernel parameter: 64 records are 13 KB of the 32 KB parameter space).
#define TFB_NOALLOC_MAX_GROUPS 64
// Size, in 32-bit words, of the allocation-free entry point's static device scratch (the
// work counter; one word used).
#define TFB_NOALLOC_SCRATCH_WORDS 64

#ifdef __cplusplus
#define TFB_EXTERN_C extern "C"
#else
#define TFB_EXTERN_C
#endif

#define TFB_GROUPED_DECLARE(set)                                                              \
  /* args: device array of tfb_group_args; items: device array of (group, tile) pairs;      \
     counter: one device word of scratch, zeroed by the launcher on `stream`.               \
     Returns a cudaError_t value. */                                                         \
  TFB_EXTERN_C int tfb_grouped_launch_##set(const void* args, const void* items,            \
                                            unsigned num_items, unsigned* counter,          \
                                            void* stream);                                  \
  /* Allocation-free form (no counterpart in the reference): for callers that cannot call   \
     cudaMalloc (code under an external memory manager that owns every device allocation,  \
     latency-critical loops where an allocation could block). host_args: num_groups         \
     tfb_group_args records in host memory (at most TFB_NOALLOC_MAX_GROUPS and the size of  \
     the fused set), passed to the kernel by value: reusable once the call returns. The     \
     work counter lives in a static device array of the library (256 bytes per GPU, kept    \
     until exit), cleared on `stream` by every call. The first call on a device looks up    \
     its address (make that call before any stream capture; the address is not refreshed   \
     after cudaDeviceReset). Calls that overlap on the GPU share the counter and race.      \
     Returns a cudaError_t value, cudaErrorInvalidValue for a null host_args or too many    \
     groups. */                                                                              \
  TFB_EXTERN_C int tfb_grouped_launch_noalloc_##set(const void* host_args,                  \
                                                    unsigned num_groups, void* stream);

#endif  // TENSORFORGE_B200_GROUPED_H
