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

#include "tnb_common.cuh"

namespace tnb {

constexpr int kGatherThreads = 256;
constexpr int kGatherEpt = TNB_GATHER_CHUNK / kGatherThreads;
constexpr int kStagedTerms = 64;

__global__ void __launch_bounds__(kGatherThreads)
gather_kernel(const int64_t* __restrict__ segs, int64_t n_seg,
              const int32_t* __restrict__ chunk_map, const int64_t* __restrict__ term_src, const double* __restrict__ term_coeff,
              const int64_t* __restrict__ term_ld, int64_t n_term,
              const double* __restrict__ src0, int64_t n_src0, double* __restrict__ dst0,
              int64_t n_dst0,
              const double* __restrict__ src1, int64_t n_src1, double* __restrict__ dst1,
              int64_t n_dst1) {
  __shared__ int64_t row[TNB_SEG_WIDTH];
  __shared__ int64_t t_src[kStagedTerms], t_ld[kStagedTerms];
  __shared__ double t_cf[kStagedTerms];
  pdl_launch_dependents();
  const int64_t chunk = blockIdx.x;
  const int64_t seg = chunk_map[chunk];
  if (seg < 0 || seg >= n_seg) {
    if (threadIdx.x == 0) raise_bounds();
    return;
  }
  if (threadIdx.x < TNB_SEG_WIDTH) row[threadIdx.x] = segs[seg * TNB_SEG_WIDTH + threadIdx.x];
  __syncthreads();

  const int64_t dst_off = row[0];
  const int64_t size = row[1];
  const int rank = static_cast<int>(row[2]);
  const int64_t t0 = row[3], t1 = row[4];
  const bool second = row[5] != 0;
  const double* __restrict__ src = second ? src1 : src0;
  double* __restrict__ dst = second ? dst1 : dst0;
  const int64_t n_src = second ? n_src1 : n_src0;
  const int64_t n_dst = second ? n_dst1 : n_dst0;
  if (t0 < 0 || t1 > n_term || t0 > t1 || rank < 1 || rank > TNB_MAX_RANK) {
    if (threadIdx.x == 0) raise_bounds();
    return;
  }
  const int nt = static_cast<int>(t1 - t0);
  const bool staged = nt <= kStagedTerms;
  if (staged && threadIdx.x < nt) {
    t_src[threadIdx.x] = term_src[t0 + threadIdx.x];
    t_ld[threadIdx.x] = term_ld[t0 + threadIdx.x];
    t_cf[threadIdx.x] = term_coeff[t0 + threadIdx.x];
  }
  __syncthreads();
  pdl_wait();  // the tables are static; the source may be the previous kernel's output

  // per-row dims and strides into registers (uniform across the CTA)
  uint32_t dims[TNB_MAX_RANK];
  int64_t dstr[TNB_MAX_RANK], rstr[TNB_MAX_RANK], cstr[TNB_MAX_RANK];
#pragma unroll
  for (int d = 0; d < TNB_MAX_RANK; ++d) {
    dims[d] = d < rank ? static_cast<uint32_t>(row[8 + d]) : 1u;
    dstr[d] = d < rank ? row[16 + d] : 0;
    rstr[d] = d < rank ? row[24 + d] : 0;
    cstr[d] = d < rank ? row[32 + d] : 0;
  }

  const int64_t base = (chunk - row[6]) * TNB_GATHER_CHUNK;
#pragma unroll
  for (int k = 0; k < kGatherEpt; ++k) {
    const int64_t e = base + threadIdx.x + k * kGatherThreads;
    if (e >= size) break;
    uint32_t rem = static_cast<uint32_t>(e);
    int64_t doff = 0, roff = 0, coff = 0;
#pragma unroll
    for (int d = TNB_MAX_RANK - 1; d >= 0; --d) {
      if (d < rank) {
        const uint32_t j = rem % dims[d];
        rem /= dims[d];
        doff += static_cast<int64_t>(j) * dstr[d];
        roff += static_cast<int64_t>(j) * rstr[d];
        coff += static_cast<int64_t>(j) * cstr[d];
      }
    }
    double acc = 0.0;
    if (staged) {
      for (int t = 0; t < nt; ++t) {
        const int64_t o = t_src[t] + t_ld[t] * roff + coff;
        if (o < 0 || o >= n_src) { raise_bounds(); continue; }
        acc = fma(t_cf[t], __ldg(src + o), acc);
      }
    } else {
      for (int64_t t = t0; t < t1; ++t) {
        const int64_t o = __ldg(term_src + t) + __ldg(term_ld + t) * roff + coff;
        if (o < 0 || o >= n_src) { raise_bounds(); continue; }
        acc = fma(__ldg(term_coeff + t), __ldg(src + o), acc);
      }
    }
    const int64_t w = dst_off + doff;
    if (w < 0 || w >= n_dst) { raise_bounds(); continue; }
    dst[w] = acc;
  }
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
  cudaError_t e = tnb::launch(tnb::gather_kernel, static_cast<unsigned>(total_chunks),
                              tnb::kGatherThreads, tnb::as_stream(stream), seg_table, n_seg,
                              chunk_map, term_src, term_coeff, term_ld, n_term, src0, n_src0,
                              dst0, n_dst0, src1, n_src1, dst1, n_dst1);
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_block_gather: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  return tnb::check_launch("tnb_block_gather");
}
