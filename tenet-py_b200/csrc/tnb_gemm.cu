// K2: grouped FP64 GEMM over the uneven coupled sectors of one composition.
//
// `compose` in the reference is one `ar.do("matmul", A_c, B_c)` per coupled sector c,
// with zeros for a sector carried by one operand only (ops/map.py:155-172).  Here every
// sector of a composition is one row of a descriptor table and the whole set runs in one
// launch: CTA b reads its (sector, tile) from a tile -> row map, so large and small
// sectors share the machine in a single wave instead of one launch each.
//
// Three tile shapes, chosen by the host per composition:
//   TNB_TILE_64     64x64 output tile, 256 threads, 4x4 register micro-tile per thread
//   TNB_TILE_32     32x32 output tile,  64 threads, same micro-tile -- for compositions
//                   whose 64x64 tiles would not fill the 148 SMs (small M, N, long K)
//   TNB_TILE_SKINNY one thread per output row, for products with N <= 16 and K <= 16
//                   (the MPO links of a matvec: tall, 1-3 columns), B staged in shared
//                   memory; bandwidth-bound by construction
// The plain form computes in FP64 on the DFMA pipe; micro-tile rows/cols are strided so
// shared-memory reads are conflict-free, and the next K slab is prefetched into
// registers while the current one is consumed.
#include <string>

#include "tnb_common.cuh"

namespace tnb {

constexpr int kBk = 16;

// Work-buffer layout of the split-K path: n_counters uint32 counters, padded to 256 bytes,
// then the FP64 partial tiles.
inline int64_t gemm_work_parts_offset(int64_t n_counters) {
  return ((4 * n_counters + 255) / 256) * 256;
}
constexpr int kSkinnyThreads = 256;
constexpr int kSkinnyMax = 16;

struct GemmRow {
  int64_t M, N, K, aoff, lda, boff, ldb, coff, ldc, tile_begin, tiles_n, splits, ksplit,
      part_off, cnt_off;
};

__device__ __forceinline__ bool load_row(const int64_t* __restrict__ table, int64_t n_gemm,
                                         const int32_t* __restrict__ tile_map, int64_t tile,
                                         GemmRow& r) {
  const int64_t g = tile_map[tile];
  if (g < 0 || g >= n_gemm) return false;
  const int64_t* t = table + g * TNB_GEMM_WIDTH;
  r.M = t[0]; r.N = t[1]; r.K = t[2]; r.aoff = t[3]; r.lda = t[4]; r.boff = t[5];
  r.ldb = t[6]; r.coff = t[7]; r.ldc = t[8]; r.tile_begin = t[9]; r.tiles_n = t[10];
  r.splits = t[12] > 1 ? t[12] : 1; r.ksplit = t[13]; r.part_off = t[14]; r.cnt_off = t[15];
  return true;
}

__device__ __forceinline__ bool footprint_ok(const GemmRow& r, int64_t n_a, int64_t n_b,
                                             int64_t n_c) {
  bool bad = r.M < 0 || r.N < 0 || r.K < 0 || r.coff < 0 || r.coff + (r.M - 1) * r.ldc + r.N > n_c;
  if (r.K > 0)
    bad = bad || r.aoff < 0 || r.boff < 0 || r.aoff + (r.M - 1) * r.lda + r.K > n_a ||
          r.boff + (r.K - 1) * r.ldb + r.N > n_b;
  return !bad;
}

template <int TM, int TN>
__global__ void __launch_bounds__((TM / 4) * (TN / 4), (TM == 64 ? 1 : 6))
gemm_f64_kernel(const int64_t* __restrict__ table, int64_t n_gemm,
                const int32_t* __restrict__ tile_map, const double* __restrict__ a,
                int64_t n_a, const double* __restrict__ b, int64_t n_b,
                double* __restrict__ c, int64_t n_c, unsigned int* __restrict__ counters,
                int64_t n_cnt, double* __restrict__ parts, int64_t n_parts) {
  constexpr int TX = TN / 4, TY = TM / 4, NT = TX * TY;
  constexpr int LA = (TM * kBk) / NT, LB = (TN * kBk) / NT;
  __shared__ double As[2][kBk][TM + 1];
  __shared__ double Bs[2][kBk][TN];
  __shared__ GemmRow s_row;
  __shared__ int s_ok;
  __shared__ int s_last;
  pdl_launch_dependents();
  const int64_t tile = blockIdx.x;
  const int tid = threadIdx.x;
  if (tid == 0) {
    GemmRow r;
    bool ok = load_row(table, n_gemm, tile_map, tile, r);
    ok = ok && footprint_ok(r, n_a, n_b, n_c);
    if (ok && r.splits > 1) {
      const int64_t nt = ((r.M + TM - 1) / TM) * r.tiles_n;
      ok = r.ksplit > 0 && r.ksplit % kBk == 0 && r.cnt_off >= 0 && r.cnt_off + nt <= n_cnt &&
           r.part_off >= 0 && r.part_off + nt * r.splits * TM * TN <= n_parts;
    }
    if (!ok) raise_bounds();
    s_row = r;
    s_ok = ok;
  }
  __syncthreads();
  if (!s_ok) return;
  const GemmRow r = s_row;
  const int64_t local = tile - r.tile_begin;
  const int64_t split = local % r.splits, t2 = local / r.splits;
  const int64_t m0 = (t2 / r.tiles_n) * TM, n0 = (t2 % r.tiles_n) * TN;
  if (m0 >= r.M || n0 >= r.N) return;
  // this CTA's K range: the whole of K, or one split of it
  const int64_t kb = r.splits > 1 ? split * r.ksplit : 0;
  const int64_t ke = r.splits > 1 ? min(r.K, kb + r.ksplit) : r.K;
  pdl_wait();  // A may be the previous kernel's output

  const int tx = tid % TX, ty = tid / TX;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;

  double ra[LA], rb[LB];
  auto load_slab = [&](int64_t k0) {
#pragma unroll
    for (int q = 0; q < LA; ++q) {
      const int idx = tid + q * NT;
      const int am = idx / kBk, ak = idx % kBk;
      const int64_t gm = m0 + am, gk = k0 + ak;
      ra[q] = (gm < r.M && gk < ke) ? __ldg(a + r.aoff + gm * r.lda + gk) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < LB; ++q) {
      const int idx = tid + q * NT;
      const int bk = idx / TN, bn = idx % TN;
      const int64_t gk = k0 + bk, gn = n0 + bn;
      rb[q] = (gk < ke && gn < r.N) ? __ldg(b + r.boff + gk * r.ldb + gn) : 0.0;
    }
  };
  auto store_slab = [&](int buf) {
#pragma unroll
    for (int q = 0; q < LA; ++q) {
      const int idx = tid + q * NT;
      As[buf][idx % kBk][idx / kBk] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < LB; ++q) {
      const int idx = tid + q * NT;
      Bs[buf][idx / TN][idx % TN] = rb[q];
    }
  };

  const int64_t nk = ke > kb ? (ke - kb + kBk - 1) / kBk : 0;
  if (nk > 0) {
    load_slab(kb);
    store_slab(0);
    __syncthreads();
  }
  for (int64_t s = 0; s < nk; ++s) {
    const int cur = static_cast<int>(s & 1);
    if (s + 1 < nk) load_slab(kb + (s + 1) * kBk);
#pragma unroll
    for (int k = 0; k < kBk; ++k) {
      double av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[cur][k][ty + TY * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[cur][k][tx + TX * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
    if (s + 1 < nk) store_slab(cur ^ 1);
    __syncthreads();
  }

  if (r.splits > 1) {
    // split K: park this partial tile, and let the last of the tile's splits to arrive
    // sum all of them in split order (a fixed order, so the result is deterministic)
    double* mine = parts + r.part_off + (t2 * r.splits + split) * (TM * TN);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) mine[(ty + TY * i) * TN + tx + TX * j] = acc[i][j];
    __threadfence();
    __syncthreads();
    if (tid == 0) {
      const unsigned int prev = atomicAdd(counters + r.cnt_off + t2, 1u);
      s_last = (prev == static_cast<unsigned int>(r.splits - 1));
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const double* base = parts + r.part_off + t2 * r.splits * (TM * TN);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int e = (ty + TY * i) * TN + tx + TX * j;
        double v = 0.0;
        for (int64_t q = 0; q < r.splits; ++q) v += __ldcg(base + q * (TM * TN) + e);
        acc[i][j] = v;
      }
    if (tid == 0) counters[r.cnt_off + t2] = 0u;  // leave the counters zero for the next run
  }

#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t gm = m0 + ty + TY * i;
    if (gm >= r.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t gn = n0 + tx + TX * j;
      if (gn < r.N) c[r.coff + gm * r.ldc + gn] = acc[i][j];
    }
  }
}

// One thread per output row: C[m, :] = A[m, :] * B for N, K <= 16.
__global__ void __launch_bounds__(kSkinnyThreads, 4)
gemm_f64_skinny_kernel(const int64_t* __restrict__ table, int64_t n_gemm,
                       const int32_t* __restrict__ tile_map, const double* __restrict__ a,
                       int64_t n_a, const double* __restrict__ b, int64_t n_b,
                       double* __restrict__ c, int64_t n_c) {
  __shared__ double Bs[kSkinnyMax * kSkinnyMax];
  __shared__ GemmRow s_row;
  __shared__ int s_ok;
  pdl_launch_dependents();
  const int64_t tile = blockIdx.x;
  const int tid = threadIdx.x;
  if (tid == 0) {
    GemmRow r;
    bool ok = load_row(table, n_gemm, tile_map, tile, r);
    ok = ok && footprint_ok(r, n_a, n_b, n_c) && r.N <= kSkinnyMax && r.K <= kSkinnyMax;
    if (!ok) raise_bounds();
    s_row = r;
    s_ok = ok;
  }
  __syncthreads();
  if (!s_ok) return;
  const GemmRow r = s_row;
  const int K = static_cast<int>(r.K), N = static_cast<int>(r.N);
  pdl_wait();  // A may be the previous kernel's output
  if (tid < K * N) Bs[tid] = __ldg(b + r.boff + (tid / N) * r.ldb + (tid % N));
  __syncthreads();
  const int64_t m = (tile - r.tile_begin) * kSkinnyThreads + tid;
  if (m >= r.M) return;
  double av[kSkinnyMax];
#pragma unroll
  for (int k = 0; k < kSkinnyMax; ++k) av[k] = k < K ? __ldg(a + r.aoff + m * r.lda + k) : 0.0;
#pragma unroll 1
  for (int n = 0; n < N; ++n) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kSkinnyMax; ++k)
      if (k < K) s = fma(av[k], Bs[k * N + n], s);
    c[r.coff + m * r.ldc + n] = s;
  }
}

}  // namespace tnb

extern "C" int tnb_grouped_gemm_f64(const int64_t* gemm_table, int64_t n_gemm,
                                    const int32_t* tile_map, int64_t total_tiles,
                                    int32_t tile_kind, const double* a, int64_t n_a,
                                    const double* b, int64_t n_b, double* c, int64_t n_c,
                                    void* work, int64_t work_bytes, int64_t n_counters,
                                    void* stream) {
  TNB_REQUIRE(n_gemm >= 0 && total_tiles >= 0, "tnb_grouped_gemm_f64: negative size");
  if (n_gemm == 0 || total_tiles == 0) return TNB_OK;
  TNB_REQUIRE(gemm_table != nullptr && tile_map != nullptr && c != nullptr,
              "tnb_grouped_gemm_f64: null table, tile map or C");
  TNB_REQUIRE(total_tiles < (int64_t(1) << 31), "tnb_grouped_gemm_f64: too many tiles");
  TNB_REQUIRE(work_bytes >= 0 && n_counters >= 0 &&
              (work_bytes == 0 || work != nullptr) &&
              tnb::gemm_work_parts_offset(n_counters) <= work_bytes,
              "tnb_grouped_gemm_f64: work buffer too small for its counters");
  auto* counters = static_cast<unsigned int*>(work);
  const int64_t poff = tnb::gemm_work_parts_offset(n_counters);
  double* parts = work_bytes > poff
                      ? reinterpret_cast<double*>(static_cast<char*>(work) + poff) : nullptr;
  const int64_t n_parts = work_bytes > poff ? (work_bytes - poff) / 8 : 0;
  const unsigned grid = static_cast<unsigned>(total_tiles);
  cudaStream_t s = tnb::as_stream(stream);
  cudaError_t e = cudaSuccess;
  switch (tile_kind) {
    case TNB_TILE_64:
      e = tnb::launch(tnb::gemm_f64_kernel<64, 64>, grid, 256, s, gemm_table, n_gemm, tile_map,
                      a, n_a, b, n_b, c, n_c, counters, n_counters, parts, n_parts);
      break;
    case TNB_TILE_32:
      e = tnb::launch(tnb::gemm_f64_kernel<32, 32>, grid, 64, s, gemm_table, n_gemm, tile_map,
                      a, n_a, b, n_b, c, n_c, counters, n_counters, parts, n_parts);
      break;
    case TNB_TILE_SKINNY:
      e = tnb::launch(tnb::gemm_f64_skinny_kernel, grid, tnb::kSkinnyThreads, s, gemm_table,
                      n_gemm, tile_map, a, n_a, b, n_b, c, n_c);
      break;
    case TNB_TILE_TC_TF32:
    case TNB_TILE_TC_3XBF16:
      e = tnb::launch_gemm_tc(tile_kind, grid, s, gemm_table, n_gemm, tile_map, a, n_a, b, n_b,
                              c, n_c);
      break;
    default:
      tnb::set_error("tnb_grouped_gemm_f64: unknown tile kind");
      return TNB_EINVAL;
  }
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_grouped_gemm_f64: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  return tnb::check_launch("tnb_grouped_gemm_f64");
}
