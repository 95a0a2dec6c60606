// Shared helpers of the tenet_b200 CUDA library: error plumbing and launch checks.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>
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

// Programmatic dependent launch.  A table-driven kernel lets the next kernel in the stream
// start as soon as every one of its CTAs is running (launch_dependents at entry), loads its
// own static tables, and only then waits for the previous kernel's results (wait).  The
// next kernel's table prologue therefore overlaps this kernel's work.  Both instructions
// are no-ops for a kernel launched without the attribute.
// Programmatic dependent launch: wait for the previous kernel's results, then let the
// next kernel launch, whose CTAs become resident and load their static tables while this
// kernel moves its data.  Releasing the next kernel at this kernel's first instruction
// instead was measured slower on the heff2 chain (49.2 against 45-47 us per matvec): the
// early dependents held SM slots this kernel's own CTAs still needed.  A kernel of many
// waves (kRelease = false) releases nothing early: its later waves would share the SMs
// with the dependents (the batched U(1)xU(1)xfZ2 update: 2.68 against 2.76 ms).  A kernel
// that returns before waiting releases its dependents when it completes.
template <bool kRelease = true>
__device__ __forceinline__ void pdl_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if constexpr (kRelease) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Whether table-driven kernels are launched with the programmatic-serialisation
// attribute (tnb_set_pdl).
bool pdl_enabled();

template <typename... KArgs, typename... Args>
cudaError_t launch(void (*kernel)(KArgs...), unsigned grid, unsigned block, cudaStream_t stream,
                   Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// The same with `smem` bytes of dynamic shared memory.
template <typename... KArgs, typename... Args>
cudaError_t launch_dyn(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem,
                       cudaStream_t stream, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Devices a process-wide per-device cache covers.
constexpr int kMaxDevices = 64;

// A kernel attribute (the dynamic shared-memory opt-in) is set per device, so a
// process that uses several GPUs must set it once on each.  `once(fn)` runs `fn` the
// first time it is called with a given device current and caches success; concurrent
// callers serialise on the mutex, and a failed attempt is retried by the next call.
class PerDeviceOnce {
 public:
  template <class F>
  cudaError_t once(F&& fn) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    if (done_[device].load(std::memory_order_acquire)) return cudaSuccess;
    std::lock_guard<std::mutex> lock(mu_);
    if (done_[device].load(std::memory_order_relaxed)) return cudaSuccess;
    e = fn();
    if (e == cudaSuccess) done_[device].store(true, std::memory_order_release);
    return e;
  }

 private:
  std::mutex mu_;
  std::atomic<bool> done_[kMaxDevices] = {};
};

// An integer attribute of the current device, computed once per device by `fn(device,
// &value)` and cached (0 when it cannot be computed, which is retried next time).
class PerDeviceInt {
 public:
  template <class F>
  int get(F&& fn) {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) {
      cudaGetLastError();
      return 0;
    }
    int v = value_[device].load(std::memory_order_acquire);
    if (v) return v;
    std::lock_guard<std::mutex> lock(mu_);
    v = value_[device].load(std::memory_order_relaxed);
    if (v) return v;
    if (fn(device, &v) != cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    value_[device].store(v, std::memory_order_release);
    return v;
  }

 private:
  std::mutex mu_;
  std::atomic<int> value_[kMaxDevices] = {};
};

// Tensor-core grouped GEMM launcher (tnb_gemm_tc.cu).
cudaError_t launch_gemm_tc(int kind, unsigned grid, cudaStream_t s, const int64_t* table,
                           int64_t n_gemm, const int32_t* tile_map, const double* a,
                           int64_t n_a, const double* b, int64_t n_b, double* c, int64_t n_c,
                           void* work, int64_t work_bytes, int64_t n_counters);

}  // namespace tnb

#define TNB_REQUIRE(cond, msg)          \
  do {                                  \
    if (!(cond)) {                      \
      tnb::set_error(msg);              \
      return TNB_EINVAL;                \
    }                                   \
  } while (0)
