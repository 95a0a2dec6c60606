// K2: grouped FP64 GEMM over the uneven coupled sectors of one composition.
//
// `compose` in the reference is one `ar.do("matmul", A_c, B_c)` per coupled sector c,
// with zeros for a sector carried by one operand only (ops/map.py:155-172).  Here every
// sector of a composition is one row of a descriptor table and the whole set runs in one
// launch: CTA b binary-searches its (sector, tile) from the rows' tile prefix, so large
// and small sectors share the machine in a single wave instead of one launch each.
//
// The plain form computes in FP64 on the DFMA pipe (sm_100a has no FP64 tcgen05 kind):
// 64x64 output tiles, BK = 16, 256 threads each holding a 4x4 register micro-tile whose
// rows/cols are strided by 16 so shared-memory reads are conflict-free, and the next
// K-slab is prefetched into registers while the current one is consumed.
#include "tnb_common.cuh"

namespace tnb {

constexpr int kTm = TNB_GEMM_TILE_M;
constexpr int kTn = TNB_GEMM_TILE_N;
constexpr int kBk = 16;
constexpr int kGemmThreads = 256;

__global__ void __launch_bounds__(kGemmThreads)
gemm_f64_kernel(const int64_t* __restrict__ table, int64_t n_gemm,
                const double* __restrict__ a, int64_t n_a, const double* __restrict__ b,
                int64_t n_b, double* __restrict__ c, int64_t n_c) {
  __shared__ double As[2][kBk][kTm + 1];
  __shared__ double Bs[2][kBk][kTn];
  __shared__ int64_t row[TNB_GEMM_WIDTH];
  __shared__ int64_t s_row;
  const int64_t tile = blockIdx.x;
  const int tid = threadIdx.x;
  if (tid == 0) {
    int64_t lo = 0, hi = n_gemm - 1;
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (table[mid * TNB_GEMM_WIDTH + 9] <= tile) lo = mid; else hi = mid - 1;
    }
    s_row = lo;
  }
  __syncthreads();
  if (tid < TNB_GEMM_WIDTH) row[tid] = table[s_row * TNB_GEMM_WIDTH + tid];
  __syncthreads();
  const int64_t M = row[0], N = row[1], K = row[2];
  const int64_t aoff = row[3], lda = row[4], boff = row[5], ldb = row[6], coff = row[7],
                ldc = row[8];
  const int64_t local = tile - row[9];
  const int64_t tm = local / row[10], tn = local % row[10];
  const int64_t m0 = tm * kTm, n0 = tn * kTn;

  // footprint check, once per CTA: a bad row raises the error word and writes nothing
  if (tid == 0) {
    bool bad = M < 0 || N < 0 || K < 0 || m0 >= M || n0 >= N || coff < 0 ||
               coff + (M - 1) * ldc + N > n_c;
    if (K > 0) bad = bad || aoff < 0 || boff < 0 || aoff + (M - 1) * lda + K > n_a ||
                     boff + (K - 1) * ldb + N > n_b;
    s_row = bad ? -1 : 0;
    if (bad) raise_bounds();
  }
  __syncthreads();
  if (s_row < 0) return;

  const int tx = tid % 16, ty = tid / 16;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;

  // loader mapping: A slab 64 x 16 (k fastest), B slab 16 x 64 (n fastest); 4 each
  double ra[4], rb[4];
  auto load_slab = [&](int64_t k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = tid + q * kGemmThreads;          // 0..1023
      const int am = idx / kBk, ak = idx % kBk;         // A: row am, col ak
      const int64_t gm = m0 + am, gk = k0 + ak;
      ra[q] = (gm < M && gk < K) ? __ldg(a + aoff + gm * lda + gk) : 0.0;
      const int bk = idx / kTn, bn = idx % kTn;          // B: row bk, col bn
      const int64_t gkb = k0 + bk, gn = n0 + bn;
      rb[q] = (gkb < K && gn < N) ? __ldg(b + boff + gkb * ldb + gn) : 0.0;
    }
  };
  auto store_slab = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = tid + q * kGemmThreads;
      As[buf][idx % kBk][idx / kBk] = ra[q];
      Bs[buf][idx / kTn][idx % kTn] = rb[q];
    }
  };

  const int64_t nk = (K + kBk - 1) / kBk;
  if (nk > 0) {
    load_slab(0);
    store_slab(0);
    __syncthreads();
  }
  for (int64_t s = 0; s < nk; ++s) {
    const int cur = static_cast<int>(s & 1);
    if (s + 1 < nk) load_slab((s + 1) * kBk);
#pragma unroll
    for (int k = 0; k < kBk; ++k) {
      double av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = As[cur][k][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = Bs[cur][k][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
    if (s + 1 < nk) store_slab(cur ^ 1);
    __syncthreads();
  }

#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t gn = n0 + tx + 16 * j;
      if (gn < N) c[coff + gm * ldc + gn] = acc[i][j];
    }
  }
}

}  // namespace tnb

extern "C" int tnb_grouped_gemm_f64(const int64_t* gemm_table, int64_t n_gemm,
                                    int64_t total_tiles, const double* a, int64_t n_a,
                                    const double* b, int64_t n_b, double* c, int64_t n_c,
                                    void* stream) {
  TNB_REQUIRE(n_gemm >= 0 && total_tiles >= 0, "tnb_grouped_gemm_f64: negative size");
  if (n_gemm == 0 || total_tiles == 0) return TNB_OK;
  TNB_REQUIRE(gemm_table != nullptr && c != nullptr, "tnb_grouped_gemm_f64: null table or C");
  TNB_REQUIRE(total_tiles < (int64_t(1) << 31), "tnb_grouped_gemm_f64: too many tiles");
  tnb::gemm_f64_kernel<<<static_cast<unsigned>(total_tiles), tnb::kGemmThreads, 0,
                         tnb::as_stream(stream)>>>(gemm_table, n_gemm, a, n_a, b, n_b, c, n_c);
  return tnb::check_launch("tnb_grouped_gemm_f64");
}
