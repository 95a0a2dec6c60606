// K3: the Lanczos vector space on a tensor arena -- qdim-weighted dot, axpby, lincomb.
//
// The reference's `inner`/`norm` are Python sums over blocks of
// `qdim(c_tau) * ar.do("sum", conj(x) * y)` (ops/contraction.py:584-589, ops/basic.py:309)
// and every Lanczos update is a per-block add (network/dmrg.py:207-227).  A tensor's
// blocks live in one contiguous arena here, so each of these is one pass over it.  The
// qdim weight is constant on runs of consecutive blocks; the host merges equal-weight
// neighbours into runs and the dot walks runs, never a per-element lookup.
#include <mutex>
#include <string>

#include "tnb_common.cuh"

namespace tnb {

constexpr int kDotThreads = 256;
constexpr int64_t kDotMaxCtas = 4 * 148;
constexpr int64_t kDotMinChunk = 2048;
// longest vector whose Lanczos step runs as one CTA (tnb_lanczos_step)
constexpr int64_t kLanczosStepMaxN = 4 * kDotMinChunk;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum in a fixed order (deterministic); the result is valid in thread 0.
__device__ double block_sum(double v) {
  __shared__ double part[kDotThreads / 32];
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = threadIdx.x < kDotThreads / 32 ? part[threadIdx.x] : 0.0;
    r = warp_sum(r);
  }
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kDotThreads)
wdot_kernel(const double* __restrict__ x, const double* __restrict__ y, int64_t n,
            const int64_t* __restrict__ run_start, const double* __restrict__ run_w,
            int64_t n_runs, int64_t chunk, unsigned int* counter, double* partial,
            double* out) {
  const int64_t lo = static_cast<int64_t>(blockIdx.x) * chunk;
  const int64_t hi = min(n, lo + chunk);
  // first run containing lo
  __shared__ int64_t s_r0;
  if (threadIdx.x == 0) {
    int64_t a = 0, b = n_runs - 1;
    while (a < b) {
      const int64_t mid = (a + b + 1) >> 1;
      if (run_start[mid] <= lo) a = mid; else b = mid - 1;
    }
    s_r0 = a;
  }
  __syncthreads();
  double acc = 0.0;
  for (int64_t r = s_r0; r < n_runs && run_start[r] < hi; ++r) {
    const int64_t a = max(lo, run_start[r]);
    const int64_t b = min(hi, run_start[r + 1]);
    double s = 0.0;
    for (int64_t i = a + threadIdx.x; i < b; i += kDotThreads) s = fma(x[i], y[i], s);
    acc = fma(run_w[r], s, acc);
  }
  const double total = block_sum(acc);
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = total;
    __threadfence();
    const unsigned int done = atomicAdd(counter, 1u);
    last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v = 0.0;
  for (int64_t i = threadIdx.x; i < gridDim.x; i += kDotThreads) v += ((volatile double*)partial)[i];
  v = block_sum(v);
  if (threadIdx.x == 0) {
    *out = v;
    *counter = 0u;  // leave the workspace reusable
  }
}

__global__ void axpby_kernel(int64_t n, double alpha, const double* x, double beta,
                             const double* y, double* out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = fma(alpha, x[i], beta * y[i]);
}

// dst[i] = src[i]: one 16-byte (or, unaligned, 8-byte) element per thread, all loads in
// flight at once, so a copy that reads or writes pinned host memory through its mapped
// pointer pays the link's latency about once.  It waits for the previous kernel first
// (its source may be that kernel's output, its destination that kernel's input).
__global__ void copy_kernel(int64_t n, const double* __restrict__ src, double* __restrict__ dst,
                            int vec) {
  pdl_wait();
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (vec) {
    if (2 * i + 1 < n) {
      reinterpret_cast<double2*>(dst)[i] = reinterpret_cast<const double2*>(src)[i];
    } else if (2 * i < n) {
      dst[2 * i] = src[2 * i];
    }
  } else if (i < n) {
    dst[i] = src[i];
  }
}

__global__ void lincomb_kernel(int64_t n, int64_t k, const double* __restrict__ coeffs,
                               const double* const* __restrict__ vecs, double* out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int64_t j = 0; j < k; ++j) s = fma(coeffs[j], vecs[j][i], s);
    out[i] = s;
  }
}

// Lanczos state on the device (doubles): [0, ncv) alpha, [ncv, 2 ncv) beta, [2 ncv, 3 ncv)
// squared norms, [3 ncv] Krylov size m, [3 ncv + 1] stopped flag.
__global__ void lanczos_update_kernel(int64_t n, double* w, const double* __restrict__ v,
                                      const double* __restrict__ vprev,
                                      const double* __restrict__ state, int j, int ncv) {
  if (state[3 * ncv + 1] != 0.0) return;  // the recurrence already stopped
  const double a = state[j];
  const double b = j > 0 ? state[ncv + j - 1] : 0.0;
  // the reference's rounding exactly: w - (v * alpha), then - (vprev * beta), each
  // product and each difference rounded on its own (no fused multiply-add)
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double x = __dsub_rn(w[i], __dmul_rn(v[i], a));
    if (j > 0) x = __dsub_rn(x, __dmul_rn(vprev[i], b));
    w[i] = x;
  }
}

__device__ __forceinline__ void lanczos_decide(const double* state, int j, int ncv, double tol,
                                               bool& live, bool& stop_now, double& beta) {
  const bool stopped = state[3 * ncv + 1] != 0.0;
  beta = sqrt(fmax(state[2 * ncv + j], 0.0));
  stop_now = !stopped && (j + 1 == ncv || beta < tol);
  live = !stopped && !stop_now;
}

// v_{j+1} = w / beta_j while the recurrence lives, zero once it stopped.  Reads the state
// only; lanczos_record_kernel (launched right after) writes the step's outcome.
__global__ void lanczos_next_kernel(int64_t n, const double* __restrict__ w, double* vnext,
                                    const double* __restrict__ state, int j, int ncv, double tol) {
  bool live, stop_now;
  double beta;
  lanczos_decide(state, j, ncv, tol, live, stop_now, beta);
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    vnext[i] = live ? __ddiv_rn(w[i], beta) : 0.0;  // w / beta, as the reference divides
}

__global__ void lanczos_record_kernel(double* state, int j, int ncv, double tol) {
  bool live, stop_now;
  double beta;
  lanczos_decide(state, j, ncv, tol, live, stop_now, beta);
  if (live) {
    state[ncv + j] = beta;
    state[3 * ncv] = static_cast<double>(j + 2);
  } else if (stop_now) {
    state[3 * ncv] = static_cast<double>(j + 1);
    state[3 * ncv + 1] = 1.0;
  }
}

// Sum of w_r * sum_i x_i y_i over the runs of [0, n), by one CTA of kDotThreads, in the
// order wdot_kernel takes over one chunk covering the whole vector (so for n up to
// kDotMinChunk -- one chunk -- the value is the standalone dot's, bit for bit).  Valid in
// every thread.
__device__ double cta_weighted_dot(const double* x, const double* y, int64_t n,
                                   const int64_t* __restrict__ run_start,
                                   const double* __restrict__ run_w, int64_t n_runs,
                                   double* bcast) {
  double acc = 0.0;
  for (int64_t r = 0; r < n_runs && run_start[r] < n; ++r) {
    const int64_t a = run_start[r];
    const int64_t b = min(n, run_start[r + 1]);
    double s = 0.0;
    for (int64_t i = a + threadIdx.x; i < b; i += kDotThreads) s = fma(x[i], y[i], s);
    acc = fma(run_w[r], s, acc);
  }
  const double total = block_sum(acc);
  if (threadIdx.x == 0) *bcast = total + 0.0;  // as the standalone dot's final reduction
  __syncthreads();
  const double v = *bcast;
  __syncthreads();
  return v;
}

// One whole step j of the recurrence after the matvec (w = H v_j) for a vector small
// enough for one CTA: alpha_j = <v_j, w>, the update, ||w||^2 and the next vector with
// the stop decision -- the work of five launches (tnb_weighted_dot, tnb_lanczos_update,
// tnb_weighted_dot, tnb_lanczos_next) in one, with the same arithmetic and state words.
__global__ void __launch_bounds__(kDotThreads)
lanczos_step_kernel(int64_t n, double* w, const double* v, const double* vprev, double* vnext,
                    double* state, int j, int ncv, double tol,
                    const int64_t* __restrict__ run_start, const double* __restrict__ run_w,
                    int64_t n_runs) {
  __shared__ double bcast;
  if (state[3 * ncv + 1] != 0.0) {  // the recurrence already stopped
    for (int64_t i = threadIdx.x; i < n; i += kDotThreads) vnext[i] = 0.0;
    return;
  }
  const double a = cta_weighted_dot(v, w, n, run_start, run_w, n_runs, &bcast);
  const double b = j > 0 ? state[ncv + j - 1] : 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kDotThreads) {
    double x = __dsub_rn(w[i], __dmul_rn(v[i], a));
    if (j > 0) x = __dsub_rn(x, __dmul_rn(vprev[i], b));
    w[i] = x;
  }
  __syncthreads();
  const double nrm2 = cta_weighted_dot(w, w, n, run_start, run_w, n_runs, &bcast);
  const double beta = sqrt(fmax(nrm2, 0.0));
  const bool stop_now = j + 1 == ncv || beta < tol;
  for (int64_t i = threadIdx.x; i < n; i += kDotThreads)
    vnext[i] = stop_now ? 0.0 : __ddiv_rn(w[i], beta);
  if (threadIdx.x == 0) {
    state[j] = a;
    state[2 * ncv + j] = nrm2;
    if (stop_now) {
      state[3 * ncv] = static_cast<double>(j + 1);
      state[3 * ncv + 1] = 1.0;
    } else {
      state[ncv + j] = beta;
      state[3 * ncv] = static_cast<double>(j + 2);
    }
  }
}

__global__ void scale_rsqrt_kernel(int64_t n, const double* __restrict__ s2, const double* x,
                                   double* out) {
  const double nrm = sqrt(s2[0]);
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = __ddiv_rn(x[i], nrm);  // x / ||x||, as the reference divides
}

// out[j] = <vecs[j], x>_qdim for j < k: one pass per j over this CTA's chunk, partials
// [j][cta] in the workspace, the last CTA reduces each j in a fixed order.
__global__ void __launch_bounds__(kDotThreads)
multi_dot_kernel(int64_t n, int64_t k, const double* const* __restrict__ vecs,
                 const double* __restrict__ x, const int64_t* __restrict__ run_start,
                 const double* __restrict__ run_w, int64_t n_runs, int64_t chunk,
                 unsigned int* counter, double* partial, double* out) {
  const int64_t lo = static_cast<int64_t>(blockIdx.x) * chunk;
  const int64_t hi = min(n, lo + chunk);
  __shared__ int64_t s_r0;
  if (threadIdx.x == 0) {
    int64_t a = 0, b = n_runs - 1;
    while (a < b) {
      const int64_t mid = (a + b + 1) >> 1;
      if (run_start[mid] <= lo) a = mid; else b = mid - 1;
    }
    s_r0 = a;
  }
  __syncthreads();
  for (int64_t j = 0; j < k; ++j) {
    const double* v = vecs[j];
    double acc = 0.0;
    for (int64_t r = s_r0; r < n_runs && run_start[r] < hi; ++r) {
      const int64_t a = max(lo, run_start[r]);
      const int64_t b = min(hi, run_start[r + 1]);
      double sum = 0.0;
      for (int64_t i = a + threadIdx.x; i < b; i += kDotThreads) sum = fma(v[i], x[i], sum);
      acc = fma(run_w[r], sum, acc);
    }
    const double total = block_sum(acc);
    if (threadIdx.x == 0) partial[j * gridDim.x + blockIdx.x] = total;
  }
  __shared__ bool last;
  if (threadIdx.x == 0) {
    __threadfence();
    last = (atomicAdd(counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int64_t j = 0; j < k; ++j) {
    double v = 0.0;
    for (int64_t i = threadIdx.x; i < gridDim.x; i += kDotThreads)
      v += ((volatile double*)partial)[j * gridDim.x + i];
    v = block_sum(v);
    if (threadIdx.x == 0) out[j] = v;
  }
  if (threadIdx.x == 0) *counter = 0u;
}

// w[i] -= sum_j coeffs[j] vecs[j][i]   (no-op once the recurrence stopped)
__global__ void reorth_kernel(int64_t n, int64_t k, const double* __restrict__ coeffs,
                              const double* const* __restrict__ vecs, double* w,
                              const double* __restrict__ state, int ncv) {
  if (state != nullptr && state[3 * ncv + 1] != 0.0) return;
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double s = 0.0;
    for (int64_t j = 0; j < k; ++j) s = fma(coeffs[j], vecs[j][i], s);
    w[i] -= s;
  }
}

inline int64_t dot_grid(int64_t n) {
  int64_t g = (n + kDotMinChunk - 1) / kDotMinChunk;
  if (g < 1) g = 1;
  if (g > kDotMaxCtas) g = kDotMaxCtas;
  return g;
}

inline unsigned elementwise_grid(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > 8 * 148) g = 8 * 148;
  return static_cast<unsigned>(g);
}

}  // namespace tnb

extern "C" int64_t tnb_dot_work_bytes(int64_t n) {
  return 256 + 8 * tnb::dot_grid(n < 0 ? 0 : n);
}

extern "C" int tnb_weighted_dot(const double* x, const double* y, int64_t n,
                                const int64_t* run_start, const double* run_w, int64_t n_runs,
                                void* work, double* out, void* stream) {
  TNB_REQUIRE(out != nullptr && work != nullptr, "tnb_weighted_dot: null out or work");
  TNB_REQUIRE(n >= 0 && n_runs >= 0, "tnb_weighted_dot: negative size");
  cudaStream_t s = tnb::as_stream(stream);
  if (n == 0 || n_runs == 0) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), s);
    if (e != cudaSuccess) {
      tnb::set_error(std::string("tnb_weighted_dot: ") + cudaGetErrorString(e));
      return TNB_ECUDA;
    }
    return TNB_OK;
  }
  TNB_REQUIRE(x != nullptr && y != nullptr && run_start != nullptr && run_w != nullptr,
              "tnb_weighted_dot: null input");
  const int64_t grid = tnb::dot_grid(n);
  const int64_t chunk = (n + grid - 1) / grid;
  auto* counter = static_cast<unsigned int*>(work);
  auto* partial = reinterpret_cast<double*>(static_cast<char*>(work) + 256);
  tnb::wdot_kernel<<<static_cast<unsigned>(grid), tnb::kDotThreads, 0, s>>>(
      x, y, n, run_start, run_w, n_runs, chunk, counter, partial, out);
  return tnb::check_launch("tnb_weighted_dot");
}

// ---------------------------------------------------------------------------------------
// Allocation-free variant of the weighted dot.  Its scratch (a counter word padded to
// 256 bytes, then one FP64 partial per CTA) is this file-scope array instead of a
// caller buffer.  Every device that loads the library holds it until the process exits.
// Each CTA reduces a fixed kNoAllocChunk elements, so the array bounds n.
namespace tnb {
constexpr int64_t kNoAllocMaxCtas = 1024;
constexpr int64_t kNoAllocChunk = 2048;
constexpr int64_t kNoAllocMaxN = kNoAllocMaxCtas * kNoAllocChunk;
static_assert(kNoAllocMaxN == TNB_DOT_NOALLOC_MAX_N, "header and kernel disagree on the limit");
static __device__ __align__(256) unsigned char g_noalloc_scratch[256 + 8 * kNoAllocMaxCtas];

// Device address of g_noalloc_scratch, looked up once per device with that device
// current.  In host code the symbol itself is only a host-side stand-in.
static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[128] = {};

// `refresh` drops the cached address first (after cudaDeviceReset the module is loaded
// again and the array may sit elsewhere).
static int noalloc_scratch(void** out, bool refresh = false) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 128) {
    set_error(std::string("tnb_weighted_dot_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (refresh) g_noalloc_ptr[dev] = nullptr;
  if (g_noalloc_ptr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error(std::string("tnb_weighted_dot_noalloc: cudaGetSymbolAddress: ") +
                cudaGetErrorString(e));
      return TNB_ECUDA;
    }
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return TNB_OK;
}
}  // namespace tnb

extern "C" int tnb_weighted_dot_noalloc(const double* x, const double* y, int64_t n,
                                        const int64_t* run_start, const double* run_w,
                                        int64_t n_runs, double* out, void* stream) {
  TNB_REQUIRE(out != nullptr, "tnb_weighted_dot_noalloc: null out");
  TNB_REQUIRE(n >= 0 && n_runs >= 0, "tnb_weighted_dot_noalloc: negative size");
  if (n > tnb::kNoAllocMaxN) {
    tnb::set_error("tnb_weighted_dot_noalloc: n = " + std::to_string(n) +
                   " exceeds the allocation-free maximum of " +
                   std::to_string(tnb::kNoAllocMaxN) +
                   " elements; use tnb_weighted_dot with caller-provided scratch");
    return TNB_EINVAL;
  }
  cudaStream_t s = tnb::as_stream(stream);
  if (n == 0 || n_runs == 0) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), s);
    if (e != cudaSuccess) {
      tnb::set_error(std::string("tnb_weighted_dot_noalloc: ") + cudaGetErrorString(e));
      return TNB_ECUDA;
    }
    return TNB_OK;
  }
  TNB_REQUIRE(x != nullptr && y != nullptr && run_start != nullptr && run_w != nullptr,
              "tnb_weighted_dot_noalloc: null input");
  void* base = nullptr;
  if (int st = tnb::noalloc_scratch(&base)) return st;
  // the counter must start at zero whatever an earlier (possibly failed) call left
  cudaError_t e = cudaMemsetAsync(base, 0, sizeof(unsigned int), s);
  if (e == cudaErrorInvalidValue || e == cudaErrorContextIsDestroyed) {
    // a stale address from before a device reset: look it up again, once
    cudaGetLastError();
    if (int st = tnb::noalloc_scratch(&base, true)) return st;
    e = cudaMemsetAsync(base, 0, sizeof(unsigned int), s);
  }
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_weighted_dot_noalloc: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  auto* counter = static_cast<unsigned int*>(base);
  auto* partial = reinterpret_cast<double*>(static_cast<char*>(base) + 256);
  const int64_t grid = (n + tnb::kNoAllocChunk - 1) / tnb::kNoAllocChunk;
  tnb::wdot_kernel<<<static_cast<unsigned>(grid), tnb::kDotThreads, 0, s>>>(
      x, y, n, run_start, run_w, n_runs, tnb::kNoAllocChunk, counter, partial, out);
  return tnb::check_launch("tnb_weighted_dot_noalloc");
}

extern "C" int tnb_lanczos_update(int64_t n, double* w, const double* v, const double* vprev,
                                  const double* state, int32_t j, int32_t ncv, void* stream) {
  TNB_REQUIRE(n >= 0 && j >= 0 && ncv > 0 && j < ncv, "tnb_lanczos_update: bad size or step");
  if (n == 0) return TNB_OK;
  TNB_REQUIRE(w && v && state && (j == 0 || vprev), "tnb_lanczos_update: null pointer");
  tnb::lanczos_update_kernel<<<tnb::elementwise_grid(n), 256, 0, tnb::as_stream(stream)>>>(
      n, w, v, vprev, state, j, ncv);
  return tnb::check_launch("tnb_lanczos_update");
}

extern "C" int tnb_lanczos_next(int64_t n, const double* w, double* vnext, double* state,
                                int32_t j, int32_t ncv, double tol, void* stream) {
  TNB_REQUIRE(n >= 0 && j >= 0 && ncv > 0 && j < ncv, "tnb_lanczos_next: bad size or step");
  TNB_REQUIRE(w && vnext && state, "tnb_lanczos_next: null pointer");
  cudaStream_t s = tnb::as_stream(stream);
  if (n > 0)
    tnb::lanczos_next_kernel<<<tnb::elementwise_grid(n), 256, 0, s>>>(n, w, vnext, state, j, ncv,
                                                                      tol);
  // stream order puts the record after every read of the state above
  tnb::lanczos_record_kernel<<<1, 1, 0, s>>>(state, j, ncv, tol);
  return tnb::check_launch("tnb_lanczos_next");
}

extern "C" int tnb_scale_rsqrt(int64_t n, const double* s2, const double* x, double* out,
                               void* stream) {
  TNB_REQUIRE(n >= 0, "tnb_scale_rsqrt: negative size");
  if (n == 0) return TNB_OK;
  TNB_REQUIRE(s2 && x && out, "tnb_scale_rsqrt: null pointer");
  tnb::scale_rsqrt_kernel<<<tnb::elementwise_grid(n), 256, 0, tnb::as_stream(stream)>>>(n, s2, x,
                                                                                       out);
  return tnb::check_launch("tnb_scale_rsqrt");
}

extern "C" int64_t tnb_multi_dot_work_bytes(int64_t n, int64_t k) {
  return 256 + 8 * tnb::dot_grid(n < 0 ? 0 : n) * (k < 1 ? 1 : k);
}

extern "C" int tnb_multi_dot(int64_t n, int64_t k, const double* const* vecs, const double* x,
                             const int64_t* run_start, const double* run_w, int64_t n_runs,
                             void* work, double* out, void* stream) {
  TNB_REQUIRE(n >= 0 && k >= 0 && n_runs >= 0, "tnb_multi_dot: negative size");
  cudaStream_t s = tnb::as_stream(stream);
  if (k == 0) return TNB_OK;
  TNB_REQUIRE(out && work, "tnb_multi_dot: null out or work");
  if (n == 0 || n_runs == 0) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * k, s);
    if (e != cudaSuccess) {
      tnb::set_error(std::string("tnb_multi_dot: ") + cudaGetErrorString(e));
      return TNB_ECUDA;
    }
    return TNB_OK;
  }
  TNB_REQUIRE(vecs && x && run_start && run_w, "tnb_multi_dot: null input");
  const int64_t grid = tnb::dot_grid(n);
  const int64_t chunk = (n + grid - 1) / grid;
  auto* counter = static_cast<unsigned int*>(work);
  auto* partial = reinterpret_cast<double*>(static_cast<char*>(work) + 256);
  tnb::multi_dot_kernel<<<static_cast<unsigned>(grid), tnb::kDotThreads, 0, s>>>(
      n, k, vecs, x, run_start, run_w, n_runs, chunk, counter, partial, out);
  return tnb::check_launch("tnb_multi_dot");
}

extern "C" int tnb_lanczos_reorth(int64_t n, int64_t k, const double* coeffs,
                                  const double* const* vecs, double* w, const double* state,
                                  int32_t ncv, void* stream) {
  TNB_REQUIRE(n >= 0 && k >= 0, "tnb_lanczos_reorth: negative size");
  if (n == 0 || k == 0) return TNB_OK;
  TNB_REQUIRE(coeffs && vecs && w, "tnb_lanczos_reorth: null pointer");
  tnb::reorth_kernel<<<tnb::elementwise_grid(n), 256, 0, tnb::as_stream(stream)>>>(
      n, k, coeffs, vecs, w, state, ncv);
  return tnb::check_launch("tnb_lanczos_reorth");
}

extern "C" int tnb_axpby(int64_t n, double alpha, const double* x, double beta, const double* y,
                         double* out, void* stream) {
  TNB_REQUIRE(n >= 0, "tnb_axpby: negative size");
  if (n == 0) return TNB_OK;
  TNB_REQUIRE(x != nullptr && y != nullptr && out != nullptr, "tnb_axpby: null pointer");
  tnb::axpby_kernel<<<tnb::elementwise_grid(n), 256, 0, tnb::as_stream(stream)>>>(n, alpha, x,
                                                                                  beta, y, out);
  return tnb::check_launch("tnb_axpby");
}

namespace {
// The address a kernel uses for `p`: device and managed memory as is, pinned host
// memory through its mapped device pointer; pageable host memory is refused (nullptr).
const void* kernel_address(const void* p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) return p;
  if (at.type == cudaMemoryTypeHost && at.devicePointer != nullptr) {
    const auto off = static_cast<const char*>(p) - static_cast<const char*>(at.hostPointer);
    return static_cast<const char*>(at.devicePointer) + off;
  }
  return nullptr;
}
}  // namespace

extern "C" int tnb_mapped_address(const void* p, void** out) {
  TNB_REQUIRE(p != nullptr && out != nullptr, "tnb_mapped_address: null pointer");
  const void* k = kernel_address(p);
  TNB_REQUIRE(k != nullptr,
              "tnb_mapped_address: neither device memory nor pinned host memory");
  *out = const_cast<void*>(k);
  return TNB_OK;
}

extern "C" int tnb_copy_f64(int64_t n, const double* src, double* dst, void* stream) {
  TNB_REQUIRE(n >= 0, "tnb_copy_f64: negative size");
  if (n == 0) return TNB_OK;
  TNB_REQUIRE(src != nullptr && dst != nullptr, "tnb_copy_f64: null pointer");
  const auto* ks = static_cast<const double*>(kernel_address(src));
  auto* kd = static_cast<double*>(const_cast<void*>(kernel_address(dst)));
  TNB_REQUIRE(ks != nullptr && kd != nullptr,
              "tnb_copy_f64: a buffer is neither device memory nor pinned host memory");
  const int vec = (reinterpret_cast<uintptr_t>(ks) % 16 == 0 &&
                   reinterpret_cast<uintptr_t>(kd) % 16 == 0) ? 1 : 0;
  const int64_t items = vec ? (n + 1) / 2 : n;
  TNB_REQUIRE(items < (int64_t(1) << 31) * 256, "tnb_copy_f64: too large for one launch");
  const cudaError_t e = tnb::launch(tnb::copy_kernel, static_cast<unsigned>((items + 255) / 256),
                                    256, tnb::as_stream(stream), n, ks, kd, vec);
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_copy_f64: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  return tnb::check_launch("tnb_copy_f64");
}

extern "C" int tnb_lincomb(int64_t n, int64_t k, const double* coeffs,
                           const double* const* vecs, double* out, void* stream) {
  TNB_REQUIRE(n >= 0 && k >= 0, "tnb_lincomb: negative size");
  if (n == 0) return TNB_OK;
  TNB_REQUIRE(out != nullptr && (k == 0 || (coeffs != nullptr && vecs != nullptr)),
              "tnb_lincomb: null pointer");
  tnb::lincomb_kernel<<<tnb::elementwise_grid(n), 256, 0, tnb::as_stream(stream)>>>(n, k, coeffs,
                                                                                    vecs, out);
  return tnb::check_launch("tnb_lincomb");
}

extern "C" int64_t tnb_lanczos_step_max_n(void) { return tnb::kLanczosStepMaxN; }

extern "C" int tnb_lanczos_step(int64_t n, double* w, const double* v, const double* vprev,
                                double* vnext, double* state, int32_t j, int32_t ncv,
                                double tol, const int64_t* run_start, const double* run_w,
                                int64_t n_runs, void* stream) {
  TNB_REQUIRE(n > 0 && n <= tnb::kLanczosStepMaxN && j >= 0 && ncv > 0 && j < ncv &&
                  n_runs > 0,
              "tnb_lanczos_step: bad size or step");
  TNB_REQUIRE(w && v && vnext && state && run_start && run_w && (j == 0 || vprev),
              "tnb_lanczos_step: null pointer");
  tnb::lanczos_step_kernel<<<1, tnb::kDotThreads, 0, tnb::as_stream(stream)>>>(
      n, w, v, vprev, vnext, state, j, ncv, tol, run_start, run_w, n_runs);
  return tnb::check_launch("tnb_lanczos_step");
}
