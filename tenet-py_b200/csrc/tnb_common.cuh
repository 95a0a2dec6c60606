// Shared helpers of the tenet_b200 CUDA library: error plumbing and launch checks.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "tenet_b200.h"

namespace tnb {

// Sticky device error word: kernels raise it (never trap) when a table-driven access
// falls outside the buffer lengths they were given.
extern __device__ int g_device_error;

__device__ __forceinline__ void raise_bounds() { atomicCAS(&g_device_error, 0, TNB_EBOUNDS); }

// Host-side error message of the last failed call on this thread.
void set_error(const std::string& msg);

int check_launch(const char* what);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace tnb

#define TNB_REQUIRE(cond, msg)          \
  do {                                  \
    if (!(cond)) {                      \
      tnb::set_error(msg);              \
      return TNB_EINVAL;                \
    }                                   \
  } while (0)
