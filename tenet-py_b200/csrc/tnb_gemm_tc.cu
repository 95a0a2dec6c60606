// K2-TC: the grouped coupled-sector GEMM on the 5th-generation tensor cores (tcgen05).
//
// The precision form of the block GEMMs: the same descriptor table as the FP64 kernels,
// FP64 operands in and FP64 results out, but every product runs as tcgen05.mma with FP32
// accumulators held in tensor memory:
//   TNB_TILE_TC_TF32    A, B rounded to TF32 (kind::tf32), one MMA per K step of 8;
//   TNB_TILE_TC_3XBF16  A = A_hi + A_lo, B = B_hi + B_lo split into BF16 pairs and the
//                       product taken as A_hi B_hi + A_hi B_lo + A_lo B_hi (kind::f16 with
//                       BF16 inputs, K step 16), which keeps about 16 significand bits of
//                       every operand instead of 8.
//
// One CTA of 128 threads owns one 128 x 64 output tile.  Per K slab of 32 the threads
// convert their share of A (128 x 32) and B (32 x 64, transposed on the way) into shared
// memory in the canonical K-major, no-swizzle UMMA layout -- 8-row x 16-byte core
// matrices, LBO = 128 B between the two core matrices of one K step, SBO between 8-row
// groups -- then one elected thread issues the MMAs into a 128-lane x 64-column TMEM
// accumulator and commits them to the stage's mbarrier.  Two shared-memory stages make a
// pipeline: slab s + 1 is loaded from global memory into registers while slab s is
// converted, stored and issued, and a stage is overwritten only after the mbarrier of
// the MMAs that read it (two slabs back) has completed.  The epilogue reads TMEM with
// tcgen05.ld (warp w owns lanes 32w..32w+31) and writes FP64.  Every wait is bounded:
// past the limit the kernel raises TNB_ETIMEOUT, stops issuing, and still frees its TMEM
// before returning.
#include <cuda_bf16.h>

#include <string>

#include "tnb_common.cuh"

namespace tnb {

constexpr int kTcM = 128, kTcN = 64, kTcBk = 32, kTcThreads = 128;
constexpr unsigned kTcTmemCols = 64;
constexpr long long kTcWaitCycles = 4000000000LL;  // ~2 s at the boost clock

struct GemmRowTc {
  int64_t M, N, K, aoff, lda, boff, ldb, coff, ldc, tile_begin, tiles_n;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor, SWIZZLE_NONE, K-major, SM100 version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) |
         (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: FP32 accumulate, both operands K-major, M = 128, N = 64.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t fmt) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((kTcN >> 3) << 17) | ((kTcM >> 4) << 24);
}

// Byte offset of element (r, k) of a K-major tile whose rows hold `row_bytes` bytes.
__device__ __forceinline__ uint32_t kmajor(int r, int k, int esz, int row_bytes) {
  const int bk = k * esz;
  return (r >> 3) * (row_bytes / 16) * 128 + (bk >> 4) * 128 + (r & 7) * 16 + (bk & 15);
}

__device__ __forceinline__ uint32_t to_tf32(double x) {
  uint32_t u;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(static_cast<float>(x)));
  return u;
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done) : "r"(mbar), "r"(phase) : "memory");
    if (done) return true;
    if (clock64() - t0 > kTcWaitCycles) return false;
  }
}

template <int MODE>
struct TcLayout {
  static constexpr int kEsz = MODE == 0 ? 4 : 2;
  static constexpr int kRowBytes = kTcBk * kEsz;
  static constexpr int kParts = MODE == 0 ? 1 : 2;
  static constexpr int kABytes = kTcM * kRowBytes, kBBytes = kTcN * kRowBytes;
  // one pipeline stage: A parts, then B parts (TF32 16 + 8 KB; 3xBF16 2 x 8 + 2 x 4 KB)
  static constexpr int kStageBytes = kParts * (kABytes + kBBytes);
  static constexpr int kSmemBytes = 2 * kStageBytes + 1024;  // two stages + alignment slack
};

template <int MODE>  // 0 = TF32, 1 = 3 x BF16
__global__ void __launch_bounds__(kTcThreads)
gemm_tc_kernel(const int64_t* __restrict__ table, int64_t n_gemm,
               const int32_t* __restrict__ tile_map, const double* __restrict__ a, int64_t n_a,
               const double* __restrict__ b, int64_t n_b, double* __restrict__ c, int64_t n_c) {
  using L = TcLayout<MODE>;
  constexpr int kEsz = L::kEsz, kRowBytes = L::kRowBytes;
  constexpr int kLA = (kTcM * kTcBk) / kTcThreads, kLB = (kTcN * kTcBk) / kTcThreads;
  extern __shared__ uint8_t smem_dyn[];
  // 1024-byte aligned base of the two stages
  uint8_t* const smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~static_cast<uintptr_t>(1023));
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t s_tmem;
  __shared__ GemmRowTc s_row;
  __shared__ int s_ok;
  __shared__ int s_fail;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  pdl_launch_dependents();
  if (tid == 0) {
    bool ok = true;
    const int64_t g = tile_map[blockIdx.x];
    GemmRowTc r{};
    if (g < 0 || g >= n_gemm) {
      ok = false;
    } else {
      const int64_t* t = table + g * TNB_GEMM_WIDTH;
      r.M = t[0]; r.N = t[1]; r.K = t[2]; r.aoff = t[3]; r.lda = t[4]; r.boff = t[5];
      r.ldb = t[6]; r.coff = t[7]; r.ldc = t[8]; r.tile_begin = t[9]; r.tiles_n = t[10];
      ok = r.M > 0 && r.N > 0 && r.K >= 0 && r.tiles_n > 0 && r.coff >= 0 &&
           r.coff + (r.M - 1) * r.ldc + r.N <= n_c;
      if (r.K > 0)
        ok = ok && r.aoff >= 0 && r.boff >= 0 && r.aoff + (r.M - 1) * r.lda + r.K <= n_a &&
             r.boff + (r.K - 1) * r.ldb + r.N <= n_b;
    }
    if (!ok) raise_bounds();
    s_row = r;
    s_ok = ok;
    s_fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[0])) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&mbar[1])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {  // one warp owns the TMEM allocation
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&s_tmem)), "r"(kTcTmemCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const GemmRowTc r = s_row;
  const bool ok = s_ok;
  const int64_t local = blockIdx.x - r.tile_begin;
  const int64_t m0 = ok ? (local / r.tiles_n) * kTcM : 0, n0 = ok ? (local % r.tiles_n) * kTcN : 0;
  pdl_wait();  // A may be the previous kernel's output

  double ra[kLA], rb[kLB];
  auto load_slab = [&](int64_t k0) {
#pragma unroll
    for (int i = 0; i < kLA; ++i) {
      const int idx = tid + i * kTcThreads;
      const int rr = idx / kTcBk, kk = idx % kTcBk;
      const int64_t gm = m0 + rr, gk = k0 + kk;
      ra[i] = (gm < r.M && gk < r.K) ? a[r.aoff + gm * r.lda + gk] : 0.0;
    }
#pragma unroll
    for (int i = 0; i < kLB; ++i) {
      const int idx = tid + i * kTcThreads;
      const int kk = idx / kTcN, nn = idx % kTcN;
      const int64_t gk = k0 + kk, gn = n0 + nn;
      rb[i] = (gk < r.K && gn < r.N) ? b[r.boff + gk * r.ldb + gn] : 0.0;
    }
  };
  auto store_slab = [&](int stage) {
    uint8_t* sa0 = smem + stage * L::kStageBytes;
    uint8_t* sb0 = sa0 + L::kParts * L::kABytes;
#pragma unroll
    for (int i = 0; i < kLA; ++i) {
      const int idx = tid + i * kTcThreads;
      const uint32_t off = kmajor(idx / kTcBk, idx % kTcBk, kEsz, kRowBytes);
      if constexpr (MODE == 0) {
        *reinterpret_cast<uint32_t*>(sa0 + off) = to_tf32(ra[i]);
      } else {
        const __nv_bfloat16 hi = __double2bfloat16(ra[i]);
        const __nv_bfloat16 lo = __double2bfloat16(ra[i] - static_cast<double>(__bfloat162float(hi)));
        *reinterpret_cast<__nv_bfloat16*>(sa0 + off) = hi;
        *reinterpret_cast<__nv_bfloat16*>(sa0 + L::kABytes + off) = lo;
      }
    }
#pragma unroll
    for (int i = 0; i < kLB; ++i) {
      const int idx = tid + i * kTcThreads;
      const uint32_t off = kmajor(idx % kTcN, idx / kTcN, kEsz, kRowBytes);
      if constexpr (MODE == 0) {
        *reinterpret_cast<uint32_t*>(sb0 + off) = to_tf32(rb[i]);
      } else {
        const __nv_bfloat16 hi = __double2bfloat16(rb[i]);
        const __nv_bfloat16 lo = __double2bfloat16(rb[i] - static_cast<double>(__bfloat162float(hi)));
        *reinterpret_cast<__nv_bfloat16*>(sb0 + off) = hi;
        *reinterpret_cast<__nv_bfloat16*>(sb0 + L::kBBytes + off) = lo;
      }
    }
  };

  uint32_t phase[2] = {0u, 0u};
  const int64_t nk = ok ? (r.K + kTcBk - 1) / kTcBk : 0;
  if (nk > 0) load_slab(0);
  for (int64_t s = 0; s < nk; ++s) {
    const int stage = static_cast<int>(s & 1);
    // the stage is free once the MMAs of slab s - 2 (its last readers) have completed
    if (s >= 2 && !s_fail && !mbar_wait(smem_u32(&mbar[stage]), phase[stage])) {
      if (lane == 0) {
        atomicCAS(&g_device_error, 0, TNB_ETIMEOUT);
        s_fail = 1;
      }
    }
    if (s >= 2) phase[stage] ^= 1u;
    __syncthreads();
    if (s_fail) break;
    store_slab(stage);
    if (s + 1 < nk) load_slab((s + 1) * kTcBk);  // in flight while slab s is issued
    // make the generic-proxy stores visible to the tensor cores, then issue
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      constexpr uint32_t kLbo = 128, kSbo = (kRowBytes / 16) * 128;
      constexpr uint32_t kIdesc = umma_idesc(MODE == 0 ? 2u : 1u);
      constexpr int kSteps = kRowBytes / 32;  // one MMA consumes 32 bytes of K
      // (A part, B part) pairs: TF32 one product; 3xBF16 hi.hi, hi.lo, lo.hi
      constexpr int kProducts = MODE == 0 ? 1 : 3;
      const int pa[3] = {0, 0, 1}, pb[3] = {0, 1, 0};
      const uint32_t sa = smem_u32(smem + stage * L::kStageBytes);
      const uint32_t sb = sa + L::kParts * L::kABytes;
#pragma unroll
      for (int p = 0; p < kProducts; ++p) {
#pragma unroll
        for (int st = 0; st < kSteps; ++st) {
          const uint64_t ad = umma_desc(sa + pa[p] * L::kABytes + st * 256, kLbo, kSbo);
          const uint64_t bd = umma_desc(sb + pb[p] * L::kBBytes + st * 256, kLbo, kSbo);
          const uint32_t acc = (s > 0 || p > 0 || st > 0) ? 1u : 0u;
          if constexpr (MODE == 0) {
            asm volatile(
                "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, q;\n\t}"
                :: "r"(tmem), "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc) : "memory");
          } else {
            asm volatile(
                "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, q;\n\t}"
                :: "r"(tmem), "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc) : "memory");
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(smem_u32(&mbar[stage])) : "memory");
    }
  }
  // the last commit covers every MMA issued before it
  if (nk > 0 && !s_fail) {
    const int last = static_cast<int>((nk - 1) & 1);
    if (!mbar_wait(smem_u32(&mbar[last]), phase[last])) {
      if (lane == 0) {
        atomicCAS(&g_device_error, 0, TNB_ETIMEOUT);
        s_fail = 1;
      }
    }
  }
  __syncthreads();

  // epilogue: TMEM -> registers -> FP64 C (zeros when K == 0 or the MMAs timed out)
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const int64_t row = m0 + warp * 32 + lane;
  const bool live = ok && nk > 0 && !s_fail;
#pragma unroll
  for (int chunk = 0; chunk < kTcN / 16; ++chunk) {
    uint32_t v[16];
    if (live) {
      const uint32_t taddr = tmem + (static_cast<uint32_t>(warp * 32) << 16) + chunk * 16;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
          "%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
            "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
            "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    } else {
#pragma unroll
      for (int j = 0; j < 16; ++j) v[j] = 0u;
    }
    if (ok && row < r.M) {
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const int64_t col = n0 + chunk * 16 + j;
        if (col < r.N) c[r.coff + row * r.ldc + col] = static_cast<double>(__uint_as_float(v[j]));
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(tmem), "r"(kTcTmemCols) : "memory");
  }
}

}  // namespace tnb

namespace tnb {
cudaError_t launch_gemm_tc(int kind, unsigned grid, cudaStream_t s, const int64_t* table,
                           int64_t n_gemm, const int32_t* tile_map, const double* a,
                           int64_t n_a, const double* b, int64_t n_b, double* c, int64_t n_c) {
  // the two-stage pipeline needs more than the default 48 KB of shared memory per CTA
  static bool opted[2] = {false, false};
  const int mode = kind == TNB_TILE_TC_TF32 ? 0 : 1;
  if (!opted[mode]) {
    const cudaError_t e = mode == 0
        ? cudaFuncSetAttribute(gemm_tc_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               TcLayout<0>::kSmemBytes)
        : cudaFuncSetAttribute(gemm_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               TcLayout<1>::kSmemBytes);
    if (e != cudaSuccess) return e;
    opted[mode] = true;
  }
  if (mode == 0)
    return launch_dyn(gemm_tc_kernel<0>, grid, kTcThreads, TcLayout<0>::kSmemBytes, s, table,
                      n_gemm, tile_map, a, n_a, b, n_b, c, n_c);
  return launch_dyn(gemm_tc_kernel<1>, grid, kTcThreads, TcLayout<1>::kSmemBytes, s, table,
                    n_gemm, tile_map, a, n_a, b, n_b, c, n_c);
}
}  // namespace tnb
