// K2-TC: the grouped coupled-sector GEMM on the 5th-generation tensor cores (tcgen05).
//
// The precision form of the block GEMMs: the same descriptor table as the FP64 kernels,
// FP64 operands in and FP64 results out, but every product runs as tcgen05.mma with FP32
// accumulators held in tensor memory:
//   TNB_TILE_TC_TF32    A, B rounded to TF32 (kind::tf32);
//   TNB_TILE_TC_3XBF16  A = A_hi + A_lo, B = B_hi + B_lo split into BF16 pairs and the
//                       product taken as A_hi B_hi + A_hi B_lo + A_lo B_hi (kind::f16 with
//                       BF16 inputs), which keeps about 16 significand bits of every
//                       operand instead of 8.
//
// Two launches per table.  A pack kernel converts each operand once: every 128-row x
// 32 slab of A (and of B^T) becomes one 16 KB chunk of the work buffer, already in the
// canonical K-major, no-swizzle UMMA shared-memory layout (8-row x 16-byte core
// matrices, LBO = 128 B between the two core matrices of one K step, SBO between 8-row
// groups), parts (BF16 hi, lo) back to back.  The MMA kernel gives each CTA a 128 x 128
// output tile and runs a three-stage pipeline: one producer thread copies the next A and
// B slabs with cp.async.bulk (global -> shared, completion counted in bytes on the
// stage's "full" mbarrier), one issuer thread waits for "full", issues the MMAs into a
// 128-lane x 128-column TMEM accumulator and commits them to the stage's "empty"
// mbarrier, which the producer waits on before refilling the stage.  The epilogue reads
// TMEM with tcgen05.ld (warp w owns lanes 32w..32w+31) and writes FP64.  Every wait is
// bounded: past the limit the kernel raises TNB_ETIMEOUT, stops, and still frees its
// TMEM before returning.  No copy uses cluster multicast.
#include <cuda_bf16.h>

#include <string>

#include "tnb_common.cuh"

namespace tnb {

constexpr int kT2M = 128, kT2N = 128, kT2Bk = 32, kT2Threads = 128, kT2Stages = 3;
constexpr int kT2Slab = 16384;  // bytes of one packed operand slab, all parts
constexpr unsigned kT2TmemCols = 128;
constexpr long long kT2WaitCycles = 4000000000LL;  // ~2 s at the boost clock

struct T2Row {
  int64_t M, N, K, aoff, lda, boff, ldb, coff, ldc, tile_begin, tiles_n, a_chunk, b_chunk;
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

// Instruction descriptor: FP32 accumulate, both operands K-major, M = 128, N = 128.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t fmt) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((kT2N >> 3) << 17) | ((kT2M >> 4) << 24);
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
    if (clock64() - t0 > kT2WaitCycles) return false;
  }
}

template <int MODE>
struct T2Layout {
  static constexpr int kEsz = MODE == 0 ? 4 : 2;
  static constexpr int kRowBytes = kT2Bk * kEsz;      // one 32-wide K row of one part
  static constexpr int kParts = MODE == 0 ? 1 : 2;
  static constexpr int kPartBytes = kT2M * kRowBytes;  // 16 KB (TF32) or 8 KB (BF16)
  static_assert(kParts * kPartBytes == kT2Slab, "a slab is 16 KB");
  static constexpr int kStageBytes = 2 * kT2Slab;      // A slab + B slab
  static constexpr int kSmemBytes = kT2Stages * kStageBytes + 1024;
};

__device__ __forceinline__ bool load_t2row(const int64_t* table, int64_t g, T2Row& r) {
  const int64_t* t = table + g * TNB_GEMM_WIDTH;
  r.M = t[0]; r.N = t[1]; r.K = t[2]; r.aoff = t[3]; r.lda = t[4]; r.boff = t[5];
  r.ldb = t[6]; r.coff = t[7]; r.ldc = t[8]; r.tile_begin = t[9]; r.tiles_n = t[10];
  r.a_chunk = t[12]; r.b_chunk = t[13];
  return r.M >= 0 && r.N >= 0 && r.K >= 0 && r.a_chunk >= 0 && r.b_chunk >= 0;
}

// The table row owning packed chunk `chunk` of operand A (which == 0) or B (which == 1):
// the last row whose first chunk is <= chunk (rows in chunk order).
__device__ int64_t owner_row(const int64_t* table, int64_t n_gemm, int64_t chunk, int which) {
  int64_t lo = 0, hi = n_gemm - 1;
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if (table[mid * TNB_GEMM_WIDTH + 12 + which] <= chunk) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Pack one 128 x 32 slab of A (blocks [0, a_chunks): rows = M, read along K) or of B^T
// (blocks after them: rows = N, read along N) into its work-buffer chunk in the UMMA
// layout.  Each of the 256 threads loads its 16 elements at once (coalesced along the
// operand's contiguous dimension), the slab is assembled in shared memory and leaves as
// 16-byte stores.
constexpr int kPackThreads = 256, kPackPer = (kT2M * kT2Bk) / kPackThreads;

template <int MODE>
__global__ void __launch_bounds__(kPackThreads)
tc_pack_kernel(const int64_t* __restrict__ table, int64_t n_gemm, const double* __restrict__ a,
               int64_t n_a, const double* __restrict__ b, int64_t n_b,
               uint8_t* __restrict__ work, int64_t work_bytes, int64_t a_chunks) {
  using L = T2Layout<MODE>;
  __shared__ __align__(16) uint8_t slab[kT2Slab];
  __shared__ T2Row s_row;
  __shared__ int s_ok;
  const int tid = threadIdx.x;
  const int which = blockIdx.x < a_chunks ? 0 : 1;
  const int64_t chunk = which == 0 ? blockIdx.x : blockIdx.x - a_chunks;
  if (tid == 0) {
    T2Row r{};
    const int64_t g = owner_row(table, n_gemm, chunk, which);
    bool ok = load_t2row(table, g, r);
    const int64_t rows = which == 0 ? r.M : r.N;
    const int64_t ks = (r.K + kT2Bk - 1) / kT2Bk;
    ok = ok && ks > 0 && (static_cast<int64_t>(blockIdx.x) + 1) * kT2Slab <= work_bytes;
    if (ok) {  // the row's operand footprint
      ok = which == 0 ? (r.aoff >= 0 && r.aoff + (r.M - 1) * r.lda + r.K <= n_a)
                      : (r.boff >= 0 && r.boff + (r.K - 1) * r.ldb + r.N <= n_b);
      ok = ok && rows > 0;
    }
    if (!ok) raise_bounds();
    s_row = r;
    s_ok = ok;
  }
  __syncthreads();
  if (!s_ok) return;
  const T2Row r = s_row;
  const int64_t ks = (r.K + kT2Bk - 1) / kT2Bk;
  const int64_t local = chunk - (which == 0 ? r.a_chunk : r.b_chunk);
  const int64_t t0 = (local / ks) * kT2M, k0 = (local % ks) * kT2Bk;
  pdl_wait();  // the operand may be the previous kernel's output
  double x[kPackPer];
#pragma unroll
  for (int i = 0; i < kPackPer; ++i) {
    const int idx = tid + i * kPackThreads;
    if (which == 0) {  // A: consecutive threads along K
      const int64_t gm = t0 + idx / kT2Bk, gk = k0 + idx % kT2Bk;
      x[i] = (gm < r.M && gk < r.K) ? __ldg(a + r.aoff + gm * r.lda + gk) : 0.0;
    } else {  // B: consecutive threads along N
      const int64_t gk = k0 + idx / kT2N, gn = t0 + idx % kT2N;
      x[i] = (gk < r.K && gn < r.N) ? __ldg(b + r.boff + gk * r.ldb + gn) : 0.0;
    }
  }
#pragma unroll
  for (int i = 0; i < kPackPer; ++i) {
    const int idx = tid + i * kPackThreads;
    const int rr = which == 0 ? idx / kT2Bk : idx % kT2N;
    const int kk = which == 0 ? idx % kT2Bk : idx / kT2N;
    const uint32_t off = kmajor(rr, kk, L::kEsz, L::kRowBytes);
    if constexpr (MODE == 0) {
      *reinterpret_cast<uint32_t*>(slab + off) = to_tf32(x[i]);
    } else {
      const __nv_bfloat16 hi = __double2bfloat16(x[i]);
      const __nv_bfloat16 lo =
          __double2bfloat16(x[i] - static_cast<double>(__bfloat162float(hi)));
      *reinterpret_cast<__nv_bfloat16*>(slab + off) = hi;
      *reinterpret_cast<__nv_bfloat16*>(slab + L::kPartBytes + off) = lo;
    }
  }
  __syncthreads();
  uint4* dst = reinterpret_cast<uint4*>(work + static_cast<int64_t>(blockIdx.x) * kT2Slab);
  const uint4* from = reinterpret_cast<const uint4*>(slab);
#pragma unroll
  for (int i = 0; i < kT2Slab / 16 / kPackThreads; ++i)
    dst[tid + i * kPackThreads] = from[tid + i * kPackThreads];
}

__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      :: "r"(dst), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}

template <int MODE>
__global__ void __launch_bounds__(kT2Threads)
tc_mma_kernel(const int64_t* __restrict__ table, int64_t n_gemm,
              const int32_t* __restrict__ tile_map, const uint8_t* __restrict__ work,
              int64_t work_bytes, int64_t b_chunk0, double* __restrict__ c, int64_t n_c) {
  using L = T2Layout<MODE>;
  extern __shared__ uint8_t smem_dyn[];
  uint8_t* const smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_dyn) + 1023) & ~static_cast<uintptr_t>(1023));
  __shared__ __align__(8) uint64_t full[kT2Stages], empty[kT2Stages], done;
  __shared__ uint32_t s_tmem;
  __shared__ T2Row s_row;
  __shared__ int s_ok, s_fail, s_fills, s_drain_fail;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    T2Row r{};
    const int64_t g = tile_map[blockIdx.x];
    bool ok = g >= 0 && g < n_gemm && load_t2row(table, g, r);
    const int64_t ks = ok ? (r.K + kT2Bk - 1) / kT2Bk : 0;
    if (ok) {
      const int64_t mt = (r.M + kT2M - 1) / kT2M, nt = (r.N + kT2N - 1) / kT2N;
      ok = r.M > 0 && r.N > 0 && r.tiles_n == nt && r.coff >= 0 &&
           r.coff + (r.M - 1) * r.ldc + r.N <= n_c &&
           (ks == 0 || ((r.a_chunk + mt * ks) * kT2Slab <= work_bytes &&
                        (b_chunk0 + r.b_chunk + nt * ks) * kT2Slab <= work_bytes));
    }
    if (!ok) raise_bounds();
    s_row = r;
    s_ok = ok;
    s_fail = 0;
    s_fills = 0;
    s_drain_fail = 0;
    for (int st = 0; st < kT2Stages; ++st) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&full[st])) : "memory");
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&empty[st])) : "memory");
    }
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(&done)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {  // one warp owns the TMEM allocation
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(&s_tmem)), "r"(kT2TmemCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  const T2Row r = s_row;
  const bool ok = s_ok;
  const int64_t local = blockIdx.x - r.tile_begin;
  const int64_t mtile = ok ? local / r.tiles_n : 0, ntile = ok ? local % r.tiles_n : 0;
  const int64_t nk = ok ? (r.K + kT2Bk - 1) / kT2Bk : 0;
  const uint8_t* a_src = work + (r.a_chunk + mtile * nk) * kT2Slab;
  const uint8_t* b_src = work + (b_chunk0 + r.b_chunk + ntile * nk) * kT2Slab;
  pdl_wait();  // the packed operands are the pack kernels' output

  if (tid == 0 && nk > 0) {  // producer
    uint32_t ephase[kT2Stages] = {0u, 0u, 0u};
    for (int64_t s = 0; s < nk; ++s) {
      const int st = static_cast<int>(s % kT2Stages);
      if (s >= kT2Stages) {
        if (!mbar_wait(smem_u32(&empty[st]), ephase[st])) {
          atomicCAS(&g_device_error, 0, TNB_ETIMEOUT);
          s_fail = 1;
          break;
        }
        ephase[st] ^= 1u;
      }
      const uint32_t fb = smem_u32(&full[st]);
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                   :: "r"(fb), "r"(static_cast<uint32_t>(2 * kT2Slab)) : "memory");
      const uint32_t sa = smem_u32(smem + st * L::kStageBytes);
      bulk_copy(sa, a_src + s * kT2Slab, kT2Slab, fb);
      bulk_copy(sa + kT2Slab, b_src + s * kT2Slab, kT2Slab, fb);
      s_fills = static_cast<int>(s + 1);
    }
  } else if (tid == 32 && nk > 0) {  // MMA issuer
    uint32_t fphase[kT2Stages] = {0u, 0u, 0u};
    constexpr uint32_t kLbo = 128, kSbo = (L::kRowBytes / 16) * 128;
    constexpr uint32_t kIdesc = umma_idesc(MODE == 0 ? 2u : 1u);
    constexpr int kSteps = L::kRowBytes / 32;  // one MMA consumes 32 bytes of K
    constexpr int kProducts = MODE == 0 ? 1 : 3;  // 3xBF16: hi.hi, hi.lo, lo.hi
    for (int64_t s = 0; s < nk; ++s) {
      const int st = static_cast<int>(s % kT2Stages);
      if (!mbar_wait(smem_u32(&full[st]), fphase[st])) {
        atomicCAS(&g_device_error, 0, TNB_ETIMEOUT);
        s_fail = 1;
        break;
      }
      fphase[st] ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sa = smem_u32(smem + st * L::kStageBytes), sb = sa + kT2Slab;
#pragma unroll
      for (int p = 0; p < kProducts; ++p) {
        const int pa = p == 2 ? 1 : 0, pb = p == 1 ? 1 : 0;
#pragma unroll
        for (int k = 0; k < kSteps; ++k) {
          const uint64_t ad = umma_desc(sa + pa * L::kPartBytes + k * 256, kLbo, kSbo);
          const uint64_t bd = umma_desc(sb + pb * L::kPartBytes + k * 256, kLbo, kSbo);
          const uint32_t acc = (s > 0 || p > 0 || k > 0) ? 1u : 0u;
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
                   :: "r"(smem_u32(&empty[st])) : "memory");
    }
    // the last commit covers every MMA issued before it
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :: "r"(smem_u32(&done)) : "memory");
  }
  __syncthreads();
  // Drain before the stages are reused and TMEM is freed, on the error path too: the
  // issuer commits `done` after whatever MMAs it issued, and every stage's last fill has
  // bulk copies that land whatever happened to the consumer.  A drain that itself gives
  // up leaves shared memory and TMEM possibly still being written, so the epilogue then
  // stores nothing.
  if (tid == 0 && nk > 0) {
    if (!mbar_wait(smem_u32(&done), 0u)) {
      atomicCAS(&g_device_error, 0, TNB_ETIMEOUT);
      s_fail = 1;
      s_drain_fail = 1;
    }
    if (s_fail) {
      const int fills = s_fills;
      for (int st = 0; st < kT2Stages && st < fills; ++st) {
        const int n_st = (fills - st + kT2Stages - 1) / kT2Stages;  // fills of stage st
        if (!mbar_wait(smem_u32(&full[st]), static_cast<uint32_t>((n_st - 1) & 1)))
          s_drain_fail = 1;
      }
    }
  }
  __syncthreads();

  // epilogue: TMEM -> registers -> shared memory -> FP64 C, 16 columns at a time (zeros
  // when K == 0 or a wait gave up).  Warp w owns TMEM lanes (tile rows) 32w..32w+31; its
  // 32 x 16 block is transposed through shared memory (the drained pipeline stages) so
  // that each store instruction writes two rows' 16 consecutive columns.
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const int64_t row0 = mtile * kT2M + warp * 32;
  const int64_t n0 = ntile * kT2N;
  const bool live = ok && nk > 0 && !s_fail;
  double* const stage = reinterpret_cast<double*>(smem) + warp * (32 * 17);
  // columns past N and warps whose rows all lie past M have nothing to store (both
  // conditions are uniform across the warp, as tcgen05.ld requires)
  const int64_t cols = ok ? r.N - n0 : 0;
  const int n_chunks = cols >= kT2N ? kT2N / 16 : static_cast<int>((cols + 15) / 16);
  const int warp_chunks = ok && row0 < r.M && !s_drain_fail ? n_chunks : 0;
#pragma unroll 1
  for (int chunk = 0; chunk < warp_chunks; ++chunk) {
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
    __syncwarp();  // the previous chunk's reads of the stage are done
#pragma unroll
    for (int j = 0; j < 16; ++j) stage[lane * 17 + j] = static_cast<double>(__uint_as_float(v[j]));
    __syncwarp();
    if (ok) {
#pragma unroll
      for (int it = 0; it < 16; ++it) {
        const int e = it * 32 + lane, rr = e >> 4, cc = e & 15;
        const int64_t row = row0 + rr, col = n0 + chunk * 16 + cc;
        if (row < r.M && col < r.N) c[r.coff + row * r.ldc + col] = stage[rr * 17 + cc];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(tmem), "r"(kT2TmemCols) : "memory");
  }
}

template <int MODE>
cudaError_t launch_tc_mode(unsigned grid, cudaStream_t s, const int64_t* table, int64_t n_gemm,
                           const int32_t* tile_map, const double* a, int64_t n_a,
                           const double* b, int64_t n_b, double* c, int64_t n_c, void* work,
                           int64_t work_bytes, int64_t a_chunks, int64_t b_chunks) {
  using L = T2Layout<MODE>;
  static PerDeviceOnce opted;
  cudaError_t e = opted.once([] {
    return cudaFuncSetAttribute(tc_mma_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                L::kSmemBytes);
  });
  if (e != cudaSuccess) return e;
  auto* w = static_cast<uint8_t*>(work);
  if (a_chunks + b_chunks > 0)
    e = launch(tc_pack_kernel<MODE>, static_cast<unsigned>(a_chunks + b_chunks), kPackThreads, s,
               table, n_gemm, a, n_a, b, n_b, w, work_bytes, a_chunks);
  if (e == cudaSuccess)
    e = launch_dyn(tc_mma_kernel<MODE>, grid, kT2Threads, L::kSmemBytes, s, table, n_gemm,
                   tile_map, static_cast<const uint8_t*>(w), work_bytes, a_chunks, c, n_c);
  return e;
}

cudaError_t launch_gemm_tc(int kind, unsigned grid, cudaStream_t s, const int64_t* table,
                           int64_t n_gemm, const int32_t* tile_map, const double* a,
                           int64_t n_a, const double* b, int64_t n_b, double* c, int64_t n_c,
                           void* work, int64_t work_bytes, int64_t n_counters) {
  const int64_t a_chunks = n_counters & 0xFFFFFFFFll, b_chunks = (n_counters >> 32) & 0xFFFFFFFFll;
  if ((a_chunks + b_chunks) * kT2Slab > work_bytes || ((a_chunks + b_chunks) > 0 && !work))
    return cudaErrorInvalidValue;
  if (kind == TNB_TILE_TC_TF32)
    return launch_tc_mode<0>(grid, s, table, n_gemm, tile_map, a, n_a, b, n_b, c, n_c, work,
                             work_bytes, a_chunks, b_chunks);
  return launch_tc_mode<1>(grid, s, table, n_gemm, tile_map, a, n_a, b, n_b, c, n_c, work,
                           work_bytes, a_chunks, b_chunks);
}

}  // namespace tnb
