// Error plumbing shared by every entry point of the tenet_b200 C ABI.
#include <cstdio>
#include <string>

#include "tnb_common.cuh"

namespace tnb {

__device__ int g_device_error = 0;

static thread_local std::string g_last_error;
static std::atomic<bool> g_pdl{true};

bool pdl_enabled() { return g_pdl.load(std::memory_order_relaxed); }

void set_error(const std::string& msg) { g_last_error = msg; }

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  return TNB_OK;
}

}  // namespace tnb

extern "C" int tnb_version(void) { return 100; }

extern "C" int tnb_set_pdl(int enabled) {
  const int prev = tnb::g_pdl.exchange(enabled != 0) ? 1 : 0;
  return prev;
}

extern "C" const char* tnb_last_error(void) { return tnb::g_last_error.c_str(); }

extern "C" int tnb_device_error(int* out, void* stream) {
  TNB_REQUIRE(out != nullptr, "tnb_device_error: out is null");
  cudaStream_t s = tnb::as_stream(stream);
  int host = 0;
  cudaError_t e = cudaMemcpyFromSymbolAsync(&host, tnb::g_device_error, sizeof(int), 0,
                                            cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && host != 0) {
    const int zero = 0;
    e = cudaMemcpyToSymbolAsync(tnb::g_device_error, &zero, sizeof(int), 0,
                                cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_device_error: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  *out = host;
  return TNB_OK;
}
