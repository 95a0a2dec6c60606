// Device bodies of the table-driven stages -- a block-gather chunk, an FP64 GEMM tile, a
// skinny GEMM tile -- shared by the standalone kernels (one launch per stage) and the
// persistent chain kernel (every stage of a compiled chain in one launch).
//
// kFused selects how data buffers are read: a standalone launch reads its sources through
// the read-only path (ld.global.nc), while inside the persistent kernel a source may have
// been written by another CTA earlier in the same launch, so it is read through L2
// (ld.global.cg), which the grid barrier's fences make coherent.  Descriptor tables never
// change during a launch and are read through the read-only path in both.
#pragma once

#include <type_traits>

#include "tnb_common.cuh"

namespace tnb {

// Synchronisation of the threads that share one work item: the whole CTA, or (several
// items per CTA in the persistent kernel) one named barrier per group of threads.
struct CtaSync {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct GroupSync {
  int id, count;
  __device__ __forceinline__ void operator()() const {
    asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(count) : "memory");
  }
};

// ---------------------------------------------------------------------------------------
// block gather

constexpr int kGatherThreads = 256;
// longest K of a product-source gather's products (the host defers only those)
constexpr int kSkinnyMaxK = 4;
constexpr int kGatherEpt = TNB_GATHER_CHUNK / kGatherThreads;
constexpr int kStagedTerms = 64;

struct GatherArgs {
  const int64_t* segs;
  int64_t n_seg;
  const int32_t* chunk_map;
  const int64_t* term_src;
  const double* term_coeff;
  const int64_t* term_ld;
  int64_t n_term;
  const double* src0;
  int64_t n_src0;
  double* dst0;
  int64_t n_dst0;
  const double* src1;
  int64_t n_src1;
  double* dst1;
  int64_t n_dst1;
  // product-source gathers only: the source is C = A x B over the GEMM table `prod`
  // (TNB_GEMM_WIDTH words per row, K <= 4); term t reads C[term_src[t] + R, term_ld[t] + C]
  // of row term_prod[t] (R, C the element's row and column strides summed)
  const int64_t* term_prod;
  const int64_t* prod;
  int64_t n_prod;
  const double* pa;
  int64_t n_pa;
  const double* pb;
  int64_t n_pb;
};

struct GatherSmem {
  int64_t row[TNB_SEG_WIDTH];
  int64_t t_src[kStagedTerms], t_ld[kStagedTerms], t_prod[kStagedTerms];
  double t_cf[kStagedTerms];
  int64_t inl[3];  // a per-chunk row's inline first term (tnb_block_gather_direct)
  int64_t dmag[TNB_MAX_RANK];  // and its extents' division constants
};

// C[m, n] of a product-source gather, computed as the FP64 GEMM kernels compute it: one
// FMA chain over k from zero, so the value is bit-identical to the materialised product.
// An element outside the product row's block, or an operand access outside A or B,
// raises the bounds error and gives 0.
__device__ __forceinline__ double product_element(const GatherArgs& g, const int64_t* pr,
                                                  int64_t m, int64_t n, bool& bad) {
  const int64_t M = __ldg(pr + 0), N = __ldg(pr + 1), K = __ldg(pr + 2), aoff = __ldg(pr + 3),
                lda = __ldg(pr + 4), boff = __ldg(pr + 5), ldb = __ldg(pr + 6);
  const int64_t a0 = aoff + m * lda, b_last = boff + (K - 1) * ldb + n;
  if (m < 0 || m >= M || n < 0 || n >= N || K > kSkinnyMaxK ||
      (K > 0 && (aoff < 0 || boff < 0 || lda < 0 || ldb < 0 || a0 + K > g.n_pa ||
                 b_last >= g.n_pb))) {
    bad = true;
    return 0.0;
  }
  double av[kSkinnyMaxK], bv[kSkinnyMaxK];
#pragma unroll
  for (int k = 0; k < kSkinnyMaxK; ++k) {
    av[k] = k < K ? __ldg(g.pa + a0 + k) : 0.0;
    bv[k] = k < K ? __ldg(g.pb + boff + k * ldb + n) : 0.0;
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kSkinnyMaxK; ++k)
    if (k < K) s = fma(av[k], bv[k], s);
  return s;
}

template <bool kFused>
__device__ __forceinline__ double load_data(const double* p) {
  if constexpr (kFused) {
    return __ldcg(p);
  } else {
    return __ldg(p);
  }
}

struct GatherElems {
  const double* __restrict__ src;
  double* __restrict__ dst;
  int64_t n_src, n_dst, dst_off, base, lim, t0, t1;
  bool staged;
};

// The KE elements base + tid + k * NT (k < KE) of one segment.  Offsets first, then the
// terms in table order, 4 / KE at a time: the four loads (terms x elements) are
// independent and in flight together, and each element still sums its terms in table
// order with one FMA chain.
template <int KE, int NT, bool kFused, bool kProd>
__device__ __forceinline__ void gather_elems(const GatherArgs& g, const GatherSmem& sm,
                                             const GatherElems& ge, int tid, int rank,
                                             const uint32_t* dims, const int64_t* dstr,
                                             const int64_t* rstr, const int64_t* cstr) {
  int64_t roff[KE], coff[KE], doff[KE];
  bool live[KE];
  double acc[KE];
#pragma unroll
  for (int k = 0; k < KE; ++k) {
    const int64_t e = ge.base + tid + k * NT;
    live[k] = e < ge.lim;
    uint32_t rem = live[k] ? static_cast<uint32_t>(e) : 0u;
    int64_t dd = 0, rr = 0, cc = 0;
#pragma unroll
    for (int d = TNB_MAX_RANK - 1; d >= 0; --d) {
      if (d < rank) {
        const uint32_t j = rem % dims[d];
        rem /= dims[d];
        dd += static_cast<int64_t>(j) * dstr[d];
        rr += static_cast<int64_t>(j) * rstr[d];
        cc += static_cast<int64_t>(j) * cstr[d];
      }
    }
    roff[k] = rr;
    coff[k] = cc;
    doff[k] = ge.dst_off + dd;
    acc[k] = 0.0;
  }
  bool bad = false;
  auto term = [&](int64_t t, int64_t& ts, int64_t& tl, double& cf, int64_t& tp) {
    if (ge.staged) {
      ts = sm.t_src[t - ge.t0];
      tl = sm.t_ld[t - ge.t0];
      cf = sm.t_cf[t - ge.t0];
      tp = kProd ? sm.t_prod[t - ge.t0] : 0;
    } else {
      ts = __ldg(g.term_src + t);
      tl = __ldg(g.term_ld + t);
      cf = __ldg(g.term_coeff + t);
      tp = kProd ? __ldg(g.term_prod + t) : 0;
    }
  };
  auto fetch = [&](int64_t ts, int64_t tl, int64_t tp, int k) -> double {
    if constexpr (kProd) {
      // term_src / term_ld hold the term's first product row and column (m0, n0): the
      // element is C[m0 + R, n0 + C] of product row tp
      if (!live[k]) return 0.0;
      if (tp < 0 || tp >= g.n_prod) {
        bad = true;
        return 0.0;
      }
      return product_element(g, g.prod + tp * TNB_GEMM_WIDTH, ts + roff[k], tl + coff[k], bad);
    } else {
      const int64_t o = ts + tl * roff[k] + coff[k];
      const bool ok = live[k] && o >= 0 && o < ge.n_src;
      bad |= live[k] && !ok;
      return ok ? load_data<kFused>(ge.src + o) : 0.0;
    }
  };
  // four loads in flight per thread (a product-source term costs 2K loads: one term)
  constexpr int kU = kProd ? 1 : (KE >= 4 ? 1 : 4 / KE);
  int64_t t = ge.t0;
  for (; t + kU <= ge.t1; t += kU) {
    int64_t ts[kU], tl[kU], tp[kU];
    double cf[kU], v[kU][KE];
#pragma unroll
    for (int u = 0; u < kU; ++u) term(t + u, ts[u], tl[u], cf[u], tp[u]);
#pragma unroll
    for (int u = 0; u < kU; ++u)
#pragma unroll
      for (int k = 0; k < KE; ++k) v[u][k] = fetch(ts[u], tl[u], tp[u], k);
#pragma unroll
    for (int u = 0; u < kU; ++u)
#pragma unroll
      for (int k = 0; k < KE; ++k) acc[k] = fma(cf[u], v[u][k], acc[k]);
  }
  for (; t < ge.t1; ++t) {
    int64_t ts, tl, tp;
    double cf, v[KE];
    term(t, ts, tl, cf, tp);
#pragma unroll
    for (int k = 0; k < KE; ++k) v[k] = fetch(ts, tl, tp, k);
#pragma unroll
    for (int k = 0; k < KE; ++k) acc[k] = fma(cf, v[k], acc[k]);
  }
#pragma unroll
  for (int k = 0; k < KE; ++k) {
    if (!live[k]) continue;
    if (doff[k] < 0 || doff[k] >= ge.n_dst) {
      bad = true;
      continue;
    }
    ge.dst[doff[k]] = acc[k];
  }
  if (bad) raise_bounds();
}

// Chunk `chunk` of the row staged in `sm` (row words, and its terms when there are at
// most kStagedTerms of them), by a group of NT threads; `tid` is the thread's index within
// the group.  Every check that depends on the row is made here, so a caller that staged
// the row ahead of time (the range kernel) gets the same validation.
template <int NT, bool kFused, bool kProd = false>
__device__ void gather_staged(const GatherArgs& g, int64_t chunk, const GatherSmem& sm,
                              int tid) {
  constexpr int kEpt = TNB_GATHER_CHUNK / NT;
  const int64_t* row = sm.row;
  const int64_t dst_off = row[0];
  const int64_t size = row[1];
  const int rank = static_cast<int>(row[2]);
  const int64_t t0 = row[3], t1 = row[4];
  const bool second = row[5] != 0;
  const double* __restrict__ src = second ? g.src1 : g.src0;
  double* __restrict__ dst = second ? g.dst1 : g.dst0;
  // (a product-source gather checks its elements against its product rows instead)
  const int64_t n_src = second ? g.n_src1 : g.n_src0;
  const int64_t n_dst = second ? g.n_dst1 : g.n_dst0;
  // the row's chunk size (a multiple of kGatherThreads up to TNB_GATHER_CHUNK)
  const int64_t ce = row[7] ? row[7] : TNB_GATHER_CHUNK;
  if (t0 < 0 || t1 > g.n_term || t0 > t1 || rank < 1 || rank > TNB_MAX_RANK ||
      (kProd && second) || ce <= 0 || ce > TNB_GATHER_CHUNK || ce % kGatherThreads ||
      chunk < row[6] || (chunk - row[6]) * ce >= size) {
    if (tid == 0) raise_bounds();
    return;
  }
  const bool staged = t1 - t0 <= kStagedTerms;

  uint32_t dims[TNB_MAX_RANK];
  int64_t dstr[TNB_MAX_RANK], rstr[TNB_MAX_RANK], cstr[TNB_MAX_RANK];
#pragma unroll
  for (int d = 0; d < TNB_MAX_RANK; ++d) {
    dims[d] = d < rank ? static_cast<uint32_t>(row[8 + d]) : 1u;
    dstr[d] = d < rank ? row[16 + d] : 0;
    rstr[d] = d < rank ? row[24 + d] : 0;
    cstr[d] = d < rank ? row[32 + d] : 0;
  }
  const int64_t base = (chunk - row[6]) * ce;
  const int64_t lim = min(size, base + ce);
  const GatherElems ge{src, dst, n_src, n_dst, dst_off, base, lim, t0, t1, staged};
  if (ce <= NT) {
    gather_elems<1, NT, kFused, kProd>(g, sm, ge, tid, rank, dims, dstr, rstr, cstr);
  } else if (ce <= 2 * NT) {
    gather_elems<(2 <= kEpt ? 2 : kEpt), NT, kFused, kProd>(g, sm, ge, tid, rank, dims, dstr,
                                                            rstr, cstr);
  } else {
    gather_elems<kEpt, NT, kFused, kProd>(g, sm, ge, tid, rank, dims, dstr, rstr, cstr);
  }
}

// Stage the terms of the row in `sm` (when there are at most kStagedTerms), one term per
// thread of the group.  False when the row's term range is invalid.
template <bool kProd>
__device__ __forceinline__ bool stage_terms(const GatherArgs& g, GatherSmem& sm, int tid) {
  const int64_t t0 = sm.row[3], t1 = sm.row[4];
  if (t0 < 0 || t1 > g.n_term || t0 > t1) return false;
  if (t1 - t0 <= kStagedTerms && tid < t1 - t0) {
    sm.t_src[tid] = g.term_src[t0 + tid];
    sm.t_ld[tid] = g.term_ld[t0 + tid];
    sm.t_cf[tid] = g.term_coeff[t0 + tid];
    if constexpr (kProd) sm.t_prod[tid] = g.term_prod[t0 + tid];
  }
  return true;
}

// One chunk of a gather with its tables staged on the spot (chunk map -> row -> terms) by
// a group of NT threads (the whole CTA standalone; a quarter of it in the persistent
// kernel); `tid` is the thread's index within the group.
template <int NT, bool kFused, class Sync, bool kProd = false, bool kRelease = true>
__device__ void gather_chunk(const GatherArgs& g, int64_t chunk, GatherSmem& sm, int tid,
                             Sync sync) {
  static_assert(!(kFused && kProd), "product-source gathers run standalone only");
  static_assert(NT >= TNB_SEG_WIDTH && NT >= kStagedTerms, "a group stages a row and its terms");
  if constexpr (kFused) sync();  // the previous item's readers are done with sm
  const int64_t seg = g.chunk_map[chunk];
  if (seg < 0 || seg >= g.n_seg) {
    if (tid == 0) raise_bounds();
    return;
  }
  if (tid < TNB_SEG_WIDTH) sm.row[tid] = g.segs[seg * TNB_SEG_WIDTH + tid];
  sync();
  const bool ok = stage_terms<kProd>(g, sm, tid);
  sync();
  if (!ok) {
    if (tid == 0) raise_bounds();
    return;
  }
  if constexpr (!kFused) pdl_wait<kRelease>();  // tables are static; the source may be the previous kernel's output
  gather_staged<NT, kFused, kProd>(g, chunk, sm, tid);
}

// Division constants of a per-chunk row (tnb_block_gather_direct): mul in the low 32 bits
// and l - 1 above them, as the host computes them (Granlund and Montgomery, "Division by
// invariant integers using multiplication", 1994: with l = ceil(log2 d) and p = 31 + l,
// mul = ceil(2^p / d) < 2^32 and mul d - 2^p < 2^(p - 31), so floor(n mul / 2^p) =
// floor(n / d) for every n < 2^31); mul = 0 stands for d = 1.

// gather_elems for a row of compile-time rank R with the row's extents, strides and
// division constants in registers: the same offsets, terms and FMA order.
template <int R, int KE, int NT>
__device__ __forceinline__ void gather_elems_rank(const GatherArgs& g, const GatherSmem& sm,
                                                  const GatherElems& ge, int tid) {
  uint32_t dims[R], mul[R], shr[R];
  int64_t dstr[R], rstr[R], cstr[R];
  // a constant is taken only if it has the property the identity needs (2^p <= mul d <
  // 2^p + 2^l with l = ceil(log2 d)); otherwise, or past 2^31 elements, hardware division
  bool mok = true;
#pragma unroll
  for (int d = 0; d < R; ++d) {
    dims[d] = static_cast<uint32_t>(sm.row[8 + d]);
    dstr[d] = sm.row[16 + d];
    rstr[d] = sm.row[24 + d];
    cstr[d] = sm.row[32 + d];
    const int64_t mag = sm.dmag[d];
    mul[d] = static_cast<uint32_t>(mag);
    const int l = static_cast<int>((mag >> 32) & 63) + 1;
    shr[d] = static_cast<uint32_t>(l - 1);
    if (dims[d] <= 1) {
      mok = mok && mul[d] == 0;
    } else {
      const bool lok = l <= 31 && l == 32 - __clz(dims[d] - 1);
      const uint64_t prod = static_cast<uint64_t>(mul[d]) * dims[d];
      const uint64_t two_p = 1ull << (lok ? 31 + l : 0);
      mok = mok && lok && prod >= two_p && prod - two_p < (1ull << l);
    }
  }
  const bool fast = mok && ge.lim <= (int64_t(1) << 31);
  int64_t roff[KE], coff[KE], doff[KE];
  bool live[KE];
  double acc[KE];
#pragma unroll
  for (int k = 0; k < KE; ++k) {
    const int64_t e = ge.base + tid + k * NT;
    live[k] = e < ge.lim;
    uint32_t rem = live[k] ? static_cast<uint32_t>(e) : 0u;
    int64_t dd = 0, rr = 0, cc = 0;
#pragma unroll
    for (int d = R - 1; d >= 0; --d) {
      const uint32_t q = fast ? (mul[d] ? __umulhi(rem, mul[d]) >> shr[d] : rem)
                              : rem / dims[d];
      const uint32_t j = rem - q * dims[d];
      rem = q;
      dd += static_cast<int64_t>(j) * dstr[d];
      rr += static_cast<int64_t>(j) * rstr[d];
      cc += static_cast<int64_t>(j) * cstr[d];
    }
    roff[k] = rr;
    coff[k] = cc;
    doff[k] = ge.dst_off + dd;
    acc[k] = 0.0;
  }
  bool bad = false;
  auto fetch = [&](int64_t ts, int64_t tl, int k) -> double {
    const int64_t o = ts + tl * roff[k] + coff[k];
    const bool ok = live[k] && o >= 0 && o < ge.n_src;
    bad |= live[k] && !ok;
    return ok ? __ldg(ge.src + o) : 0.0;
  };
  const bool one = ge.t1 - ge.t0 == 1;
  auto term = [&](int64_t t, int64_t& ts, int64_t& tl, double& cf) {
    if (one) {
      ts = sm.inl[0];
      cf = __longlong_as_double(static_cast<long long>(sm.inl[1]));
      tl = sm.inl[2];
    } else if (ge.staged) {
      ts = sm.t_src[t - ge.t0];
      tl = sm.t_ld[t - ge.t0];
      cf = sm.t_cf[t - ge.t0];
    } else {
      ts = __ldg(g.term_src + t);
      tl = __ldg(g.term_ld + t);
      cf = __ldg(g.term_coeff + t);
    }
  };
  // four loads in flight per thread, as gather_elems
  constexpr int kU = KE >= 4 ? 1 : 4 / KE;
  int64_t t = ge.t0;
  for (; t + kU <= ge.t1; t += kU) {
    int64_t ts[kU], tl[kU];
    double cf[kU], v[kU][KE];
#pragma unroll
    for (int u = 0; u < kU; ++u) term(t + u, ts[u], tl[u], cf[u]);
#pragma unroll
    for (int u = 0; u < kU; ++u)
#pragma unroll
      for (int k = 0; k < KE; ++k) v[u][k] = fetch(ts[u], tl[u], k);
#pragma unroll
    for (int u = 0; u < kU; ++u)
#pragma unroll
      for (int k = 0; k < KE; ++k) acc[k] = fma(cf[u], v[u][k], acc[k]);
  }
  for (; t < ge.t1; ++t) {
    int64_t ts, tl;
    double cf, v[KE];
    term(t, ts, tl, cf);
#pragma unroll
    for (int k = 0; k < KE; ++k) v[k] = fetch(ts, tl, k);
#pragma unroll
    for (int k = 0; k < KE; ++k) acc[k] = fma(cf, v[k], acc[k]);
  }
#pragma unroll
  for (int k = 0; k < KE; ++k) {
    if (!live[k]) continue;
    if (doff[k] < 0 || doff[k] >= ge.n_dst) {
      bad = true;
      continue;
    }
    ge.dst[doff[k]] = acc[k];
  }
  if (bad) raise_bounds();
}

// The chunk of a per-chunk row staged in `sm` (row, terms, division constants): the checks
// of gather_staged, then gather_elems_rank for the row's rank (1 to kDirectMaxRank; the
// host sends tables with higher ranks to tnb_block_gather).
constexpr int kDirectMaxRank = 4;

template <int NT>
__device__ void gather_direct_staged(const GatherArgs& g, int64_t chunk, const GatherSmem& sm,
                                     int tid) {
  constexpr int kEpt = TNB_GATHER_CHUNK / NT;
  const int64_t* row = sm.row;
  const int rank = static_cast<int>(row[2]);
  const int64_t size = row[1], t0 = row[3], t1 = row[4];
  const bool second = row[5] != 0;
  const int64_t ce = row[7] ? row[7] : TNB_GATHER_CHUNK;
  if (t0 < 0 || t1 > g.n_term || t0 > t1 || rank < 1 || rank > kDirectMaxRank || ce <= 0 ||
      ce > TNB_GATHER_CHUNK ||
      ce % kGatherThreads || chunk < row[6] || (chunk - row[6]) * ce >= size) {
    if (tid == 0) raise_bounds();
    return;
  }
  const int64_t base = (chunk - row[6]) * ce;
  const GatherElems ge{second ? g.src1 : g.src0, second ? g.dst1 : g.dst0,
                       second ? g.n_src1 : g.n_src0, second ? g.n_dst1 : g.n_dst0, row[0],
                       base, min(size, base + ce), t0, t1, t1 - t0 <= kStagedTerms};
  auto run = [&](auto rank_tag) {
    constexpr int R = decltype(rank_tag)::value;
    if (ce <= NT) {
      gather_elems_rank<R, 1, NT>(g, sm, ge, tid);
    } else if (ce <= 2 * NT) {
      gather_elems_rank<R, (2 <= kEpt ? 2 : kEpt), NT>(g, sm, ge, tid);
    } else {
      gather_elems_rank<R, kEpt, NT>(g, sm, ge, tid);
    }
  };
  switch (rank) {
    case 1: run(std::integral_constant<int, 1>{}); break;
    case 2: run(std::integral_constant<int, 2>{}); break;
    case 3: run(std::integral_constant<int, 3>{}); break;
    default: run(std::integral_constant<int, 4>{}); break;
  }
}

// word of a per-chunk row where its extents' division constants begin
constexpr int kChunkRowMagic = 48;

// CP consecutive chunks first, first + 1, ... (those below `total`) of a gather whose table
// is a row per chunk (TNB_CHUNK_ROW_WIDTH words: the segment row, its first term inline,
// its extents' division constants), by one CTA: every chunk's row -- and, for a one-term
// row, its term -- arrives in the same round of independent loads (a 64-thread group
// per chunk), so the CTA waits on its table once for CP chunks; rows with more terms
// stage them in a second round.  The chunks then run one after the other.  The loads of
// the static table come before the dependent-launch wait.
template <int NT, int CP, bool kRelease = true>
__device__ void gather_chunks_direct(const GatherArgs& g, const int64_t* __restrict__ crows,
                                     int64_t first, int64_t total, GatherSmem* sm, int tid) {
  static_assert(TNB_CHUNK_ROW_WIDTH <= 64 && CP * 64 <= NT && NT >= kStagedTerms,
                "a 64-thread group stages each chunk row");
  {
    const int i = tid / 64, w = tid % 64;
    if (i < CP && first + i < total) {
      const int64_t* cr = crows + (first + i) * TNB_CHUNK_ROW_WIDTH;
      GatherSmem& c = sm[i];
      if (w < TNB_SEG_WIDTH) {
        c.row[w] = __ldg(cr + w);
      } else if (w < TNB_SEG_WIDTH + 3) {
        c.inl[w - TNB_SEG_WIDTH] = __ldg(cr + w);
      } else if (w >= kChunkRowMagic && w < kChunkRowMagic + TNB_MAX_RANK) {
        c.dmag[w - kChunkRowMagic] = __ldg(cr + w);
      }
    }
  }
  __syncthreads();
  // a one-term row's term is read from the inline words where it is used; rows with more
  // terms stage them (every condition here is uniform across the CTA, so is the barrier)
  bool ok[CP], staged = false;
#pragma unroll
  for (int i = 0; i < CP; ++i) {
    ok[i] = false;
    if (first + i >= total) continue;
    GatherSmem& c = sm[i];
    const int64_t t0 = c.row[3], t1 = c.row[4];
    ok[i] = t0 >= 0 && t1 <= g.n_term && t0 <= t1;
    if (!ok[i]) {
      if (tid == 0) raise_bounds();
    } else if (t1 - t0 > 1) {
      if (t1 - t0 <= kStagedTerms && tid < t1 - t0) {
        c.t_src[tid] = __ldg(g.term_src + t0 + tid);
        c.t_ld[tid] = __ldg(g.term_ld + t0 + tid);
        c.t_cf[tid] = __ldg(g.term_coeff + t0 + tid);
      }
      staged = true;
    }
  }
  if (staged) __syncthreads();
  pdl_wait<kRelease>();  // the source may be the previous kernel's output
#pragma unroll
  for (int i = 0; i < CP; ++i)
    if (ok[i]) gather_direct_staged<NT>(g, first + i, sm[i], tid);
}

// ---------------------------------------------------------------------------------------
// grouped FP64 GEMM tiles

constexpr int kBk = 16;
constexpr int kSkinnyThreads = 256;
constexpr int kSkinnyMax = 16;

// Work-buffer layout of the split-K path: n_counters uint32 counters, padded to 256 bytes,
// then the FP64 partial tiles.
__host__ __device__ inline int64_t gemm_work_parts_offset(int64_t n_counters) {
  return ((4 * n_counters + 255) / 256) * 256;
}

struct GemmArgs {
  const int64_t* table;
  int64_t n_gemm;
  const int32_t* tile_map;
  const double* a;
  int64_t n_a;
  const double* b;
  int64_t n_b;
  double* c;
  int64_t n_c;
  unsigned int* counters;
  int64_t n_cnt;
  double* parts;
  int64_t n_parts;
  // when set, the table as one row per tile (tnb_grouped_gemm_f64_rows): tile t's row at
  // tile_rows + t * TNB_GEMM_WIDTH, no tile map to read first
  const int64_t* tile_rows;
};

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

__device__ __forceinline__ bool load_row(const GemmArgs& g, int64_t tile, GemmRow& r) {
  if (g.tile_rows == nullptr) return load_row(g.table, g.n_gemm, g.tile_map, tile, r);
  if (tile < 0 || tile >= g.n_gemm) return false;  // n_gemm holds the tile count here
  const int64_t* t = g.tile_rows + tile * TNB_GEMM_WIDTH;
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

// S K slabs of both operands.  The persistent chain kernel uses S = 2 with the next slab
// prefetched through registers (its sources may have been written earlier in the same
// launch and are read through L2); a standalone launch keeps S - 1 slabs in flight with
// cp.async (operands are fixed for the launch), which the DFMA loop needs at the few warps
// per SM that small coupled sectors give.
template <int TM, int TN, int S = 2>
struct GemmSmem {
  double As[S][kBk][TM + 1];
  double Bs[S][kBk][TN];
  GemmRow row;
  int ok;
  int last;
};

__device__ __forceinline__ void cp_async8(void* smem_dst, const double* src, bool ok) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;"
               :: "r"(static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst))), "l"(src),
                  "r"(ok ? 8u : 0u) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory");
}

// One TM x TN output tile (or one K split of it) by the NT = TM*TN/16 threads of a group;
// `tid` is the thread's index within the group.
template <int TM, int TN, bool kFused, class Sync, int S>
__device__ void gemm_tile(const GemmArgs& g, int64_t tile, GemmSmem<TM, TN, S>& sm, int tid,
                          Sync sync) {
  static_assert(!kFused || S == 2, "the persistent kernel double-buffers through registers");
  constexpr int TX = TN / 4, TY = TM / 4, NT = TX * TY;
  constexpr int LA = (TM * kBk) / NT, LB = (TN * kBk) / NT;
  if constexpr (kFused) sync();  // the previous item's readers are done with sm
  if (tid == 0) {
    GemmRow r;
    bool ok = load_row(g, tile, r);
    ok = ok && footprint_ok(r, g.n_a, g.n_b, g.n_c);
    if (ok && r.splits > 1) {
      const int64_t nt = ((r.M + TM - 1) / TM) * r.tiles_n;
      ok = r.ksplit > 0 && r.ksplit % kBk == 0 && r.cnt_off >= 0 && r.cnt_off + nt <= g.n_cnt &&
           r.part_off >= 0 && r.part_off + nt * r.splits * TM * TN <= g.n_parts;
    }
    if (!ok) raise_bounds();
    sm.row = r;
    sm.ok = ok;
  }
  sync();
  if (!sm.ok) return;
  const GemmRow r = sm.row;
  const int64_t local = tile - r.tile_begin;
  const int64_t split = local % r.splits, t2 = local / r.splits;
  const int64_t m0 = (t2 / r.tiles_n) * TM, n0 = (t2 % r.tiles_n) * TN;
  if (m0 >= r.M || n0 >= r.N) return;
  const int64_t kb = r.splits > 1 ? split * r.ksplit : 0;
  const int64_t ke = r.splits > 1 ? min(r.K, kb + r.ksplit) : r.K;
  if constexpr (!kFused) pdl_wait();  // A may be the previous kernel's output

  const double* __restrict__ a = g.a;
  const double* __restrict__ b = g.b;
  const int tx = tid % TX, ty = tid / TX;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;

  auto slab_fma = [&](int buf) {
#pragma unroll
    for (int k = 0; k < kBk; ++k) {
      double av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = sm.As[buf][k][ty + TY * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = sm.Bs[buf][k][tx + TX * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
  };
  const int64_t nk = ke > kb ? (ke - kb + kBk - 1) / kBk : 0;

  if constexpr (kFused) {
  double ra[LA], rb[LB];
  auto load_slab = [&](int64_t k0) {
#pragma unroll
    for (int q = 0; q < LA; ++q) {
      const int idx = tid + q * NT;
      const int am = idx / kBk, ak = idx % kBk;
      const int64_t gm = m0 + am, gk = k0 + ak;
      ra[q] = (gm < r.M && gk < ke) ? load_data<kFused>(a + r.aoff + gm * r.lda + gk) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < LB; ++q) {
      const int idx = tid + q * NT;
      const int bk = idx / TN, bn = idx % TN;
      const int64_t gk = k0 + bk, gn = n0 + bn;
      rb[q] = (gk < ke && gn < r.N) ? load_data<kFused>(b + r.boff + gk * r.ldb + gn) : 0.0;
    }
  };
  auto store_slab = [&](int buf) {
#pragma unroll
    for (int q = 0; q < LA; ++q) {
      const int idx = tid + q * NT;
      sm.As[buf][idx % kBk][idx / kBk] = ra[q];
    }
#pragma unroll
    for (int q = 0; q < LB; ++q) {
      const int idx = tid + q * NT;
      sm.Bs[buf][idx / TN][idx % TN] = rb[q];
    }
  };

  if (nk > 0) {
    load_slab(kb);
    store_slab(0);
    sync();
  }
  for (int64_t s = 0; s < nk; ++s) {
    const int cur = static_cast<int>(s & 1);
    if (s + 1 < nk) load_slab(kb + (s + 1) * kBk);
    slab_fma(cur);
    if (s + 1 < nk) store_slab(cur ^ 1);
    sync();
  }
  } else {
  // slab s lands in buffer s % S; S - 1 slabs are in flight while one is consumed
  const double* const a0 = a + r.aoff;
  const double* const b0 = b + r.boff;
  auto issue = [&](int64_t s) {
    const int buf = static_cast<int>(s % S);
    const int64_t k0 = kb + s * kBk;
#pragma unroll
    for (int q = 0; q < LA; ++q) {
      const int idx = tid + q * NT;
      const int am = idx / kBk, ak = idx % kBk;
      const int64_t gm = m0 + am, gk = k0 + ak;
      const bool ok = gm < r.M && gk < ke;
      cp_async8(&sm.As[buf][ak][am], ok ? a0 + gm * r.lda + gk : a0, ok);
    }
#pragma unroll
    for (int q = 0; q < LB; ++q) {
      const int idx = tid + q * NT;
      const int bk = idx / TN, bn = idx % TN;
      const int64_t gk = k0 + bk, gn = n0 + bn;
      const bool ok = gk < ke && gn < r.N;
      cp_async8(&sm.Bs[buf][bk][bn], ok ? b0 + gk * r.ldb + gn : b0, ok);
    }
  };
#pragma unroll
  for (int s = 0; s < S - 1; ++s) {
    if (s < nk) issue(s);
    cp_async_commit();
  }
  for (int64_t s = 0; s < nk; ++s) {
    cp_async_wait<S - 2>();  // this thread's copies of slab s have landed
    sync();                  // everyone's have, and slab s - 1 is consumed
    if (s + S - 1 < nk) issue(s + S - 1);
    cp_async_commit();
    slab_fma(static_cast<int>(s % S));
  }
  cp_async_wait<0>();
  }

  if (r.splits > 1) {
    // split K: park this partial tile, and let the last of the tile's splits to arrive
    // sum all of them in split order (a fixed order, so the result is deterministic)
    double* mine = g.parts + r.part_off + (t2 * r.splits + split) * (TM * TN);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) mine[(ty + TY * i) * TN + tx + TX * j] = acc[i][j];
    __threadfence();
    sync();
    if (tid == 0) {
      const unsigned int prev = atomicAdd(g.counters + r.cnt_off + t2, 1u);
      sm.last = (prev == static_cast<unsigned int>(r.splits - 1));
    }
    sync();
    if (!sm.last) return;
    __threadfence();
    const double* base = g.parts + r.part_off + t2 * r.splits * (TM * TN);
    // splits outermost: each element still sums its splits in split order from zero, and
    // the 16 loads of one split are in flight together
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    for (int64_t q = 0; q < r.splits; ++q) {
      double v[4][4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
          v[i][j] = __ldcg(base + q * (TM * TN) + (ty + TY * i) * TN + tx + TX * j);
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] += v[i][j];
    }
    if (tid == 0) g.counters[r.cnt_off + t2] = 0u;  // leave the counters zero for the next run
  }

#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int64_t gm = m0 + ty + TY * i;
    if (gm >= r.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int64_t gn = n0 + tx + TX * j;
      if (gn < r.N) g.c[r.coff + gm * r.ldc + gn] = acc[i][j];
    }
  }
}

struct SkinnySmem {
  double Bs[kSkinnyMax * kSkinnyMax];
  GemmRow row;
  int ok;
};

// kSkinnyThreads output rows, C[m, :] = A[m, :] * B for N, K <= 16, by a group of NT
// threads (one row each standalone; kSkinnyThreads / NT rows each in the persistent
// kernel, which gives every thread independent loads to overlap).
template <int NT, bool kFused, class Sync>
__device__ void skinny_tile(const GemmArgs& g, int64_t tile, SkinnySmem& sm, int tid, Sync sync) {
  constexpr int kRows = kSkinnyThreads / NT;
  if constexpr (kFused) sync();
  if (tid == 0) {
    GemmRow r;
    bool ok = load_row(g, tile, r);
    ok = ok && footprint_ok(r, g.n_a, g.n_b, g.n_c) && r.N <= kSkinnyMax && r.K <= kSkinnyMax;
    if (!ok) raise_bounds();
    sm.row = r;
    sm.ok = ok;
  }
  sync();
  if (!sm.ok) return;
  const GemmRow r = sm.row;
  const int K = static_cast<int>(r.K), N = static_cast<int>(r.N);
  if constexpr (!kFused) pdl_wait();  // A may be the previous kernel's output
  for (int i = tid; i < K * N; i += NT)
    sm.Bs[i] = load_data<kFused>(g.b + r.boff + (i / N) * r.ldb + (i % N));
  sync();
  const int64_t m_base = (tile - r.tile_begin) * kSkinnyThreads + tid;
  // rows in batches of up to two: both rows' loads are issued before either is used
  constexpr int kBatch = kRows < 2 ? kRows : 2;
#pragma unroll 1
  for (int q0 = 0; q0 < kRows; q0 += kBatch) {
    double av[kBatch][kSkinnyMax];
#pragma unroll
    for (int q = 0; q < kBatch; ++q) {
      const int64_t m = m_base + (q0 + q) * NT;
#pragma unroll
      for (int k = 0; k < kSkinnyMax; ++k)
        av[q][k] = (m < r.M && k < K) ? load_data<kFused>(g.a + r.aoff + m * r.lda + k) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < kBatch; ++q) {
      const int64_t m = m_base + (q0 + q) * NT;
      if (m >= r.M) break;
#pragma unroll 1
      for (int n = 0; n < N; ++n) {
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < kSkinnyMax; ++k)
          if (k < K) s = fma(av[q][k], sm.Bs[k * N + n], s);
        g.c[r.coff + m * r.ldc + n] = s;
      }
    }
  }
}

// kSkinnyThreads output columns, C[:, n] = A * B[:, n] for M, K <= 16, one column per
// thread (the transpose of the skinny case: a few rows, a long N): A is staged in shared
// memory, and loads of B and stores of C run along N, so both are coalesced.
__device__ inline void wide_tile(const GemmArgs& g, int64_t tile, SkinnySmem& sm) {
  const int tid = threadIdx.x;
  if (tid == 0) {
    GemmRow r;
    bool ok = load_row(g, tile, r);
    ok = ok && footprint_ok(r, g.n_a, g.n_b, g.n_c) && r.M <= kSkinnyMax && r.K <= kSkinnyMax;
    if (!ok) raise_bounds();
    sm.row = r;
    sm.ok = ok;
  }
  __syncthreads();
  if (!sm.ok) return;
  const GemmRow r = sm.row;
  const int M = static_cast<int>(r.M), K = static_cast<int>(r.K);
  pdl_wait();  // B may be the previous kernel's output
  for (int i = tid; i < M * K; i += kSkinnyThreads)
    sm.Bs[i] = __ldg(g.a + r.aoff + (i / K) * r.lda + (i % K));
  __syncthreads();
  const int64_t n = (tile - r.tile_begin) * kSkinnyThreads + tid;
  if (n >= r.N) return;
  double bv[kSkinnyMax];
#pragma unroll
  for (int k = 0; k < kSkinnyMax; ++k) bv[k] = k < K ? __ldg(g.b + r.boff + k * r.ldb + n) : 0.0;
#pragma unroll 1
  for (int m = 0; m < M; ++m) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kSkinnyMax; ++k)
      if (k < K) s = fma(sm.Bs[m * K + k], bv[k], s);
    g.c[r.coff + m * r.ldc + n] = s;
  }
}

}  // namespace tnb
