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
//   TNB_TILE_WIDE   one thread per output column, for products with M <= 16 and K <= 16
//                   (an MPO tensor as the left operand: a few rows, a long N)
// The plain form computes in FP64 on the DFMA pipe; micro-tile rows/cols are strided so
// shared-memory reads are conflict-free, and the next K slabs stream into shared memory
// with cp.async (three ahead for 32 x 32 tiles, two for 64 x 64) while one is consumed.
#include <string>

#include "tnb_stages.cuh"

namespace tnb {

// K slabs in shared memory per tile shape: 32 x 32 keeps three in flight (33 KB, six CTAs
// per SM), 64 x 64 two (50 KB, dynamic shared memory).
template <int TM>
constexpr int kGemmStages = TM == 64 ? 3 : 4;

template <int TM, int TN>
__global__ void __launch_bounds__((TM / 4) * (TN / 4), (TM == 64 ? 1 : 6))
gemm_f64_kernel(const GemmArgs g) {
  extern __shared__ __align__(16) uint8_t gemm_smem[];
  auto& sm = *reinterpret_cast<GemmSmem<TM, TN, kGemmStages<TM>>*>(gemm_smem);
  gemm_tile<TM, TN, false>(g, blockIdx.x, sm, threadIdx.x, CtaSync{});
}

template <int TM, int TN>
cudaError_t launch_gemm_f64(unsigned grid, cudaStream_t s, const GemmArgs& g) {
  constexpr size_t kSmem = sizeof(GemmSmem<TM, TN, kGemmStages<TM>>);
  static PerDeviceOnce opted;
  const cudaError_t e = opted.once([] {
    return cudaFuncSetAttribute(gemm_f64_kernel<TM, TN>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem);
  });
  if (e != cudaSuccess) return e;
  return launch_dyn(gemm_f64_kernel<TM, TN>, grid, (TM / 4) * (TN / 4), kSmem, s, g);
}

__global__ void __launch_bounds__(kSkinnyThreads, 4)
gemm_f64_skinny_kernel(const GemmArgs g) {
  __shared__ SkinnySmem sm;
  skinny_tile<kSkinnyThreads, false>(g, blockIdx.x, sm, threadIdx.x, CtaSync{});
}

__global__ void __launch_bounds__(kSkinnyThreads, 4)
gemm_f64_wide_kernel(const GemmArgs g) {
  __shared__ SkinnySmem sm;
  wide_tile(g, blockIdx.x, sm);
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
  const bool tc = tile_kind == TNB_TILE_TC_TF32 || tile_kind == TNB_TILE_TC_3XBF16;
  TNB_REQUIRE(work_bytes >= 0 && n_counters >= 0 && (work_bytes == 0 || work != nullptr),
              "tnb_grouped_gemm_f64: bad work buffer");
  TNB_REQUIRE(tc || tnb::gemm_work_parts_offset(n_counters) <= work_bytes,
              "tnb_grouped_gemm_f64: work buffer too small for its counters");
  TNB_REQUIRE(!tc || ((n_counters & 0xFFFFFFFFll) + (n_counters >> 32)) * 16384 <= work_bytes,
              "tnb_grouped_gemm_f64: work buffer too small for the packed operands");
  auto* counters = static_cast<unsigned int*>(work);
  const int64_t poff = tnb::gemm_work_parts_offset(n_counters);
  double* parts = work_bytes > poff
                      ? reinterpret_cast<double*>(static_cast<char*>(work) + poff) : nullptr;
  const int64_t n_parts = work_bytes > poff ? (work_bytes - poff) / 8 : 0;
  const unsigned grid = static_cast<unsigned>(total_tiles);
  cudaStream_t s = tnb::as_stream(stream);
  cudaError_t e = cudaSuccess;
  const tnb::GemmArgs g{gemm_table, n_gemm, tile_map, a, n_a, b, n_b, c, n_c, counters,
                        n_counters, parts, n_parts};
  switch (tile_kind) {
    case TNB_TILE_64:
      e = tnb::launch_gemm_f64<64, 64>(grid, s, g);
      break;
    case TNB_TILE_32:
      e = tnb::launch_gemm_f64<32, 32>(grid, s, g);
      break;
    case TNB_TILE_SKINNY:
      e = tnb::launch(tnb::gemm_f64_skinny_kernel, grid, tnb::kSkinnyThreads, s, g);
      break;
    case TNB_TILE_WIDE:
      e = tnb::launch(tnb::gemm_f64_wide_kernel, grid, tnb::kSkinnyThreads, s, g);
      break;
    case TNB_TILE_TC_TF32:
    case TNB_TILE_TC_3XBF16:
      e = tnb::launch_gemm_tc(tile_kind, grid, s, gemm_table, n_gemm, tile_map, a, n_a, b, n_b,
                              c, n_c, work, work_bytes, n_counters);
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

extern "C" int tnb_grouped_gemm_f64_rows(const int64_t* tile_rows, int64_t total_tiles,
                                         int32_t tile_kind, const double* a, int64_t n_a,
                                         const double* b, int64_t n_b, double* c, int64_t n_c,
                                         void* work, int64_t work_bytes, int64_t n_counters,
                                         void* stream) {
  TNB_REQUIRE(total_tiles >= 0, "tnb_grouped_gemm_f64_rows: negative size");
  if (total_tiles == 0) return TNB_OK;
  TNB_REQUIRE(tile_rows != nullptr && c != nullptr, "tnb_grouped_gemm_f64_rows: null rows or C");
  TNB_REQUIRE(total_tiles < (int64_t(1) << 31), "tnb_grouped_gemm_f64_rows: too many tiles");
  TNB_REQUIRE(tile_kind == TNB_TILE_64 || tile_kind == TNB_TILE_32 ||
                  tile_kind == TNB_TILE_SKINNY || tile_kind == TNB_TILE_WIDE,
              "tnb_grouped_gemm_f64_rows: FP64 tile kinds only");
  TNB_REQUIRE(work_bytes >= 0 && n_counters >= 0 && (work_bytes == 0 || work != nullptr) &&
                  tnb::gemm_work_parts_offset(n_counters) <= work_bytes,
              "tnb_grouped_gemm_f64_rows: bad work buffer");
  auto* counters = static_cast<unsigned int*>(work);
  const int64_t poff = tnb::gemm_work_parts_offset(n_counters);
  double* parts = work_bytes > poff
                      ? reinterpret_cast<double*>(static_cast<char*>(work) + poff) : nullptr;
  const int64_t n_parts = work_bytes > poff ? (work_bytes - poff) / 8 : 0;
  const unsigned grid = static_cast<unsigned>(total_tiles);
  cudaStream_t s = tnb::as_stream(stream);
  const tnb::GemmArgs g{nullptr, total_tiles, nullptr, a, n_a, b, n_b, c, n_c, counters,
                        n_counters, parts, n_parts, tile_rows};
  cudaError_t e = cudaSuccess;
  switch (tile_kind) {
    case TNB_TILE_64:
      e = tnb::launch_gemm_f64<64, 64>(grid, s, g);
      break;
    case TNB_TILE_32:
      e = tnb::launch_gemm_f64<32, 32>(grid, s, g);
      break;
    case TNB_TILE_SKINNY:
      e = tnb::launch(tnb::gemm_f64_skinny_kernel, grid, tnb::kSkinnyThreads, s, g);
      break;
    default:
      e = tnb::launch(tnb::gemm_f64_wide_kernel, grid, tnb::kSkinnyThreads, s, g);
      break;
  }
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_grouped_gemm_f64_rows: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  return tnb::check_launch("tnb_grouped_gemm_f64_rows");
}
