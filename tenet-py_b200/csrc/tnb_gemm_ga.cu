// K2-GA: a grouped FP64 GEMM whose A operand is gathered where it is read.
//
// In a compiled chain every product C_c = A_c B_c of a link is preceded by a gather that
// builds the packed A_c from the previous product (or the chain's input): the permute,
// bend and to_matrices of the reference (ops/repartition.py:458-476, map_view.py:238-279),
// then compose's matmul (ops/map.py:155-172).  Here one launch does both: the gather is
// given as a per-element list of terms (CSR over the packed A: for element e, terms
// [a_ptr[e], a_ptr[e+1]) of (source offset, coefficient), in the gather's own term
// order), and each CTA evaluates the A elements of its tile straight into shared memory
// -- acc = fma(coefficient, source, acc) from zero, exactly the gather's arithmetic --
// before the same FMA chain over K as the FP64 tiles.  No packed A is written or read
// back, and the link is one launch instead of two.
//
// For the small products of a DMRG matvec at small bonds: K <= kGaMaxK, 32 x 32 output
// tiles, no split-K, at most kGaMaxTerms terms per tile.  The tile's CSR row pointers and
// terms are static and staged in shared memory before the programmatic-dependent-launch
// wait; after it, one round of independent loads fetches every term's source value and
// B, and each A element is summed from shared memory.
#include <string>

#include "tnb_stages.cuh"

namespace tnb {

constexpr int kGaTM = 32, kGaTN = 32, kGaThreads = 256, kGaMaxK = 128;
// terms of one tile's A elements staged in shared memory (the host admits a link only
// when every tile fits)
constexpr int kGaMaxTerms = 5120;

struct GaSmem {
  double A[kGaTM][kGaMaxK + 1];
  double B[kGaMaxK][kGaTN];
  double cf[kGaMaxTerms];
  double val[kGaMaxTerms];
  int32_t src[kGaMaxTerms];
  int32_t ptr[kGaTM * kGaMaxK + 1];
  GemmRow row;
  int ok;
};

struct GaArgs {
  GemmArgs g;  // table, tile map, (unused a), b, c
  const int32_t* a_ptr;
  int64_t n_ptr;  // entries of a_ptr (packed A elements + 1)
  const int32_t* a_src;
  const double* a_cf;
  int64_t n_terms;
  const double* src;
  int64_t n_src;
};

__global__ void __launch_bounds__(kGaThreads)
gemm_ga_kernel(const GaArgs ga) {
  extern __shared__ __align__(16) unsigned char ga_smem[];
  GaSmem& sm = *reinterpret_cast<GaSmem*>(ga_smem);
  const GemmArgs& g = ga.g;
  const int tid = threadIdx.x;
  if (tid == 0) {
    GemmRow r;
    bool ok = load_row(g.table, g.n_gemm, g.tile_map, blockIdx.x, r);
    ok = ok && r.M >= 0 && r.N >= 0 && r.K >= 0 && r.K <= kGaMaxK && r.coff >= 0 &&
         (r.M == 0 || r.N == 0 || r.coff + (r.M - 1) * r.ldc + r.N <= g.n_c);
    if (ok && r.K > 0 && r.M > 0 && r.N > 0)
      ok = r.lda == r.K && r.aoff >= 0 && r.aoff + r.M * r.K < ga.n_ptr && r.boff >= 0 &&
           r.boff + (r.K - 1) * r.ldb + r.N <= g.n_b;
    if (!ok) raise_bounds();
    sm.row = r;
    sm.ok = ok;
  }
  __syncthreads();
  if (!sm.ok) return;
  const GemmRow r = sm.row;
  const int64_t local = blockIdx.x - r.tile_begin;
  const int64_t m0 = (local / r.tiles_n) * kGaTM, n0 = (local % r.tiles_n) * kGaTN;
  const int K = static_cast<int>(r.K);
  const int rows = static_cast<int>(r.M - m0 < kGaTM ? r.M - m0 : kGaTM);
  const int cols = static_cast<int>(r.N - n0 < kGaTN ? r.N - n0 : kGaTN);
  if (rows <= 0 || cols <= 0) return;  // uniform across the CTA
  const int ne = rows * K;
  // static, before the wait: the tile's CSR row pointers, then its terms (a contiguous
  // range of the term arrays: elements and their terms are both in packed-A order)
  const int64_t e0 = r.aoff + m0 * K;
  if (K > 0)
    for (int i = tid; i <= ne; i += kGaThreads) sm.ptr[i] = __ldg(ga.a_ptr + e0 + i);
  __syncthreads();
  const int32_t tb = K > 0 ? sm.ptr[0] : 0, te = K > 0 ? sm.ptr[ne] : 0;
  const int nt = te - tb;
  const bool terms_ok = tb >= 0 && nt >= 0 && nt <= kGaMaxTerms && te <= ga.n_terms;
  if (terms_ok)
    for (int i = tid; i < nt; i += kGaThreads) {
      sm.src[i] = __ldg(ga.a_src + tb + i);
      sm.cf[i] = __ldg(ga.a_cf + tb + i);
    }
  pdl_wait();  // the source is the previous kernel's output
  __syncthreads();
  bool bad = !terms_ok;
  // every term's source value in one round of independent loads; then each element
  // sums its terms in their order, from zero, as the gather does
  if (terms_ok)
    for (int i = tid; i < nt; i += kGaThreads) {
      const int64_t o = sm.src[i];
      const bool ok = o >= 0 && o < ga.n_src;
      bad |= !ok;
      sm.val[i] = ok ? __ldg(ga.src + o) : 0.0;
    }
  for (int i = tid; i < K * kGaTN; i += kGaThreads) {
    const int k = i / kGaTN, n = i % kGaTN;
    sm.B[k][n] = n < cols ? __ldg(g.b + r.boff + static_cast<int64_t>(k) * r.ldb + n0 + n) : 0.0;
  }
  __syncthreads();
  for (int i = tid; i < ne; i += kGaThreads) {
    double acc = 0.0;
    if (terms_ok) {
      const int t0 = sm.ptr[i] - tb, t1 = sm.ptr[i + 1] - tb;
      if (t0 < 0 || t1 < t0 || t1 > nt) {
        bad = true;
      } else {
        for (int t = t0; t < t1; ++t) acc = fma(sm.cf[t], sm.val[t], acc);
      }
    }
    sm.A[i / K][i % K] = acc;
  }
  if (bad) raise_bounds();
  __syncthreads();
  // 256 threads x (2 rows x 2 columns): row ty + 16 i, column tx + 16 j
  const int tx = tid % 16, ty = tid / 16;
  double acc[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (int k = 0; k < K; ++k) {
    const double a0 = sm.A[ty][k], a1 = sm.A[ty + 16][k];
    const double b0 = sm.B[k][tx], b1 = sm.B[k][tx + 16];
    acc[0][0] = fma(a0, b0, acc[0][0]);
    acc[0][1] = fma(a0, b1, acc[0][1]);
    acc[1][0] = fma(a1, b0, acc[1][0]);
    acc[1][1] = fma(a1, b1, acc[1][1]);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int m = ty + 16 * i;
    if (m >= rows) continue;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int n = tx + 16 * j;
      if (n < cols) g.c[r.coff + (m0 + m) * r.ldc + n0 + n] = acc[i][j];
    }
  }
}

static PerDeviceOnce g_ga_opt;

}  // namespace tnb

extern "C" int tnb_grouped_gemm_gather_a(const int64_t* gemm_table, int64_t n_gemm,
                                         const int32_t* tile_map, int64_t total_tiles,
                                         const int32_t* a_ptr, int64_t n_ptr,
                                         const int32_t* a_src, const double* a_cf,
                                         int64_t n_terms, const double* src, int64_t n_src,
                                         const double* b, int64_t n_b, double* c, int64_t n_c,
                                         void* stream) {
  TNB_REQUIRE(n_gemm >= 0 && total_tiles >= 0 && n_ptr >= 0 && n_terms >= 0 && n_src >= 0 &&
                  n_b >= 0 && n_c >= 0, "tnb_grouped_gemm_gather_a: negative size");
  if (n_gemm == 0 || total_tiles == 0) return TNB_OK;
  TNB_REQUIRE(gemm_table && tile_map && a_ptr && c && (n_terms == 0 || (a_src && a_cf)) &&
                  (n_src == 0 || src) && (n_b == 0 || b),
              "tnb_grouped_gemm_gather_a: null pointer");
  TNB_REQUIRE(total_tiles < (int64_t(1) << 31) && n_terms < (int64_t(1) << 31),
              "tnb_grouped_gemm_gather_a: too many tiles or terms");
  cudaError_t e = tnb::g_ga_opt.once([] {
    return cudaFuncSetAttribute(tnb::gemm_ga_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(sizeof(tnb::GaSmem)));
  });
  const tnb::GaArgs ga{{gemm_table, n_gemm, tile_map, nullptr, 0, b, n_b, c, n_c, nullptr, 0,
                        nullptr, 0},
                       a_ptr, n_ptr, a_src, a_cf, n_terms, src, n_src};
  if (e == cudaSuccess)
    e = tnb::launch_dyn(tnb::gemm_ga_kernel, static_cast<unsigned>(total_tiles), tnb::kGaThreads,
                        sizeof(tnb::GaSmem), tnb::as_stream(stream), ga);
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_grouped_gemm_gather_a: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  return tnb::check_launch("tnb_grouped_gemm_gather_a");
}
