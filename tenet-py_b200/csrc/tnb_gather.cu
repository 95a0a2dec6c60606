// K1: table-driven block gather -- permute, scale by the fusion-tree coefficient, sum
// the terms of one destination block, write once.
//
// One launch executes a whole block map: every (destination block, source terms) row of
// a transpose / bend / repartition plan, or of the block <-> coupled-sector-matrix
// lowering.  The reference runs the same map as a Python loop of one `ar.do("transpose")`
// per source block plus one scaled add per term (ops/repartition.py:458-476,
// map_view.py:266-279, map_view.py:323-334).  Here each destination region is owned by
// one row, so the sum over terms happens in registers: no atomics, no pre-zeroing, and a
// fixed summation order (the order of the terms in the plan), hence deterministic.
//
// Work is cut into TNB_GATHER_CHUNK-element chunks; CTA b reads its row index from a
// chunk -> row map (one load, no search), stages the row and up to kStagedTerms terms in
// shared memory, then streams its elements.  The kernel is HBM-bound: algorithmic bytes per element
// are 8 * (terms + 1).  A source term may be a strided window of a coupled-sector matrix
// with its own leading dimension (see the row layout in tenet_b200.h).
#include <string>

#include "tnb_stages.cuh"

namespace tnb {

// Two builds of one kernel.  Three CTAs per SM (72 registers, no spills) for tables of up
// to two waves of chunks, where each CTA's latency matters; four (64 registers, a few
// spilled) for larger tables, where more resident warps keep more loads in flight
// (measured on the batched U(1)xU(1)xfZ2 update: 2.02 against 2.27 ms for its gathers;
// on the single heff2 matvec's one-wave gathers the three-CTA build is as fast or faster).
// The four-CTA build, always many waves, does not release the next kernel early.
template <int kMinBlocks>
__global__ void __launch_bounds__(kGatherThreads, kMinBlocks)
gather_kernel(const GatherArgs g) {
  __shared__ GatherSmem sm;
  gather_chunk<kGatherThreads, false, CtaSync, false, (kMinBlocks == 3)>(g, blockIdx.x, sm,
                                                                         threadIdx.x, CtaSync{});
}

// The per-chunk-row form (tnb_block_gather_direct), the same two builds.
// (The many-wave build takes kDirectChunksPerCta chunks per CTA: one table wait for both.
// Measured on the config-3 batch: 1.66 ms of gathers with one chunk per CTA, 1.51 with
// two, 1.60 with three, 1.68 with four -- fewer resident CTAs per chunk in flight; two
// per CTA in the three-CTA-per-SM build (80 registers, no spills) took 1.71.)
constexpr int kDirectChunksPerCta = 2;

template <int kMinBlocks, int CP>
__global__ void __launch_bounds__(kGatherThreads, kMinBlocks)
gather_direct_kernel(const GatherArgs g, const int64_t* __restrict__ chunk_rows, int64_t total) {
  __shared__ GatherSmem sm[CP];
  gather_chunks_direct<kGatherThreads, CP, (kMinBlocks == 3)>(
      g, chunk_rows, static_cast<int64_t>(blockIdx.x) * CP, total, sm, threadIdx.x);
}

// SMs of the current device (0 when it cannot be queried), cached per device.
int device_sms() {
  static PerDeviceInt cached;
  return cached.get([](int device, int* v) {
    return cudaDeviceGetAttribute(v, cudaDevAttrMultiProcessorCount, device);
  });
}

// The product-source form: every source element is an element of C = A x B of a GEMM
// table with K <= 4 (an MPO link), computed where it is read instead of being written by
// a GEMM launch and read back.  Two CTAs per SM: the product's 2K operand loads per term need
// the registers.
__global__ void __launch_bounds__(kGatherThreads, 2)
gather_product_kernel(const GatherArgs g) {
  __shared__ GatherSmem sm;
  gather_chunk<kGatherThreads, false, CtaSync, true>(g, blockIdx.x, sm, threadIdx.x, CtaSync{});
}

}  // namespace tnb

extern "C" int tnb_block_gather(const int64_t* seg_table, int64_t n_seg, const int32_t* chunk_map,
                                int64_t total_chunks,
                                const int64_t* term_src, const double* term_coeff,
                                const int64_t* term_ld, int64_t n_term, const double* src0, int64_t n_src0, double* dst0, int64_t n_dst0,
                                const double* src1, int64_t n_src1, double* dst1, int64_t n_dst1,
                                void* stream) {
  TNB_REQUIRE(n_seg >= 0 && total_chunks >= 0 && n_term >= 0, "tnb_block_gather: negative size");
  if (n_seg == 0 || total_chunks == 0) return TNB_OK;
  TNB_REQUIRE(seg_table != nullptr && chunk_map != nullptr,
              "tnb_block_gather: seg_table or chunk_map is null");
  TNB_REQUIRE(n_term == 0 || (term_src != nullptr && term_coeff != nullptr && term_ld != nullptr),
              "tnb_block_gather: term arrays are null");
  TNB_REQUIRE(dst0 != nullptr || dst1 != nullptr, "tnb_block_gather: no destination buffer");
  TNB_REQUIRE(total_chunks < (int64_t(1) << 31), "tnb_block_gather: too many chunks for one launch");
  const tnb::GatherArgs g{seg_table, n_seg, chunk_map, term_src, term_coeff, term_ld, n_term,
                          src0, n_src0, dst0, n_dst0, src1, n_src1, dst1, n_dst1};
  const bool large = total_chunks > 2 * 3 * static_cast<int64_t>(tnb::device_sms());
  cudaError_t e = large ? tnb::launch(tnb::gather_kernel<4>, static_cast<unsigned>(total_chunks),
                                      tnb::kGatherThreads, tnb::as_stream(stream), g)
                        : tnb::launch(tnb::gather_kernel<3>, static_cast<unsigned>(total_chunks),
                                      tnb::kGatherThreads, tnb::as_stream(stream), g);
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_block_gather: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  return tnb::check_launch("tnb_block_gather");
}

extern "C" int tnb_block_gather_product(const int64_t* seg_table, int64_t n_seg,
                                        const int32_t* chunk_map, int64_t total_chunks,
                                        const int64_t* term_src, const double* term_coeff,
                                        const int64_t* term_ld, const int64_t* term_prod,
                                        int64_t n_term, const int64_t* prod_table,
                                        int64_t n_prod, const double* a, int64_t n_a,
                                        const double* b, int64_t n_b, double* dst,
                                        int64_t n_dst, void* stream) {
  TNB_REQUIRE(n_seg >= 0 && total_chunks >= 0 && n_term >= 0 && n_prod >= 0 && n_a >= 0 &&
                  n_b >= 0 && n_dst >= 0,
              "tnb_block_gather_product: negative size");
  if (n_seg == 0 || total_chunks == 0) return TNB_OK;
  TNB_REQUIRE(seg_table != nullptr && chunk_map != nullptr && dst != nullptr,
              "tnb_block_gather_product: seg_table, chunk_map or dst is null");
  TNB_REQUIRE(n_term == 0 || (term_src != nullptr && term_coeff != nullptr &&
                              term_ld != nullptr && term_prod != nullptr),
              "tnb_block_gather_product: term arrays are null");
  TNB_REQUIRE(n_prod > 0 && prod_table != nullptr && a != nullptr && b != nullptr,
              "tnb_block_gather_product: no product table or operands");
  TNB_REQUIRE(total_chunks < (int64_t(1) << 31),
              "tnb_block_gather_product: too many chunks for one launch");
  tnb::GatherArgs g{seg_table, n_seg, chunk_map, term_src, term_coeff, term_ld, n_term,
                    nullptr, 0, dst, n_dst, nullptr, 0, nullptr, 0};
  g.term_prod = term_prod;
  g.prod = prod_table;
  g.n_prod = n_prod;
  g.pa = a;
  g.n_pa = n_a;
  g.pb = b;
  g.n_pb = n_b;
  cudaError_t e = tnb::launch(tnb::gather_product_kernel, static_cast<unsigned>(total_chunks),
                              tnb::kGatherThreads, tnb::as_stream(stream), g);
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_block_gather_product: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  return tnb::check_launch("tnb_block_gather_product");
}

extern "C" int tnb_block_gather_direct(const int64_t* chunk_rows, int64_t total_chunks,
                                       const int64_t* term_src, const double* term_coeff,
                                       const int64_t* term_ld, int64_t n_term,
                                       const double* src0, int64_t n_src0, double* dst0,
                                       int64_t n_dst0, const double* src1, int64_t n_src1,
                                       double* dst1, int64_t n_dst1, void* stream) {
  TNB_REQUIRE(total_chunks >= 0 && n_term >= 0, "tnb_block_gather_direct: negative size");
  if (total_chunks == 0) return TNB_OK;
  TNB_REQUIRE(chunk_rows != nullptr, "tnb_block_gather_direct: chunk_rows is null");
  TNB_REQUIRE(n_term == 0 || (term_src != nullptr && term_coeff != nullptr && term_ld != nullptr),
              "tnb_block_gather_direct: term arrays are null");
  TNB_REQUIRE(dst0 != nullptr || dst1 != nullptr, "tnb_block_gather_direct: no destination buffer");
  TNB_REQUIRE(total_chunks < (int64_t(1) << 31),
              "tnb_block_gather_direct: too many chunks for one launch");
  const tnb::GatherArgs g{nullptr, 0, nullptr, term_src, term_coeff, term_ld, n_term,
                          src0, n_src0, dst0, n_dst0, src1, n_src1, dst1, n_dst1};
  const bool large = total_chunks > 2 * 3 * static_cast<int64_t>(tnb::device_sms());
  constexpr int CP = tnb::kDirectChunksPerCta;
  cudaError_t e =
      large ? tnb::launch(tnb::gather_direct_kernel<4, CP>,
                          static_cast<unsigned>((total_chunks + CP - 1) / CP), tnb::kGatherThreads,
                          tnb::as_stream(stream), g, chunk_rows, total_chunks)
            : tnb::launch(tnb::gather_direct_kernel<3, 1>, static_cast<unsigned>(total_chunks),
                          tnb::kGatherThreads, tnb::as_stream(stream), g, chunk_rows,
                          total_chunks);
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_block_gather_direct: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  return tnb::check_launch("tnb_block_gather_direct");
}
