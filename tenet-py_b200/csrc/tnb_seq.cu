// Recorded launch sequences and the native Lanczos driver.
//
// A sequence is a list of table-driven launches (gathers and grouped GEMMs) recorded
// once, with their tables, buffers and sizes, and replayed by one call.  Replay can
// substitute buffer pointers (a compiled matvec is recorded on placeholder input and
// output buffers and replayed on the Krylov vectors), so one recorded chain program
// serves every matvec of a solve without host work per launch.  The Lanczos driver
// launches a whole solve -- ncv matvecs, the recurrence, optional FP64
// reorthogonalisation -- from one host call; nothing in it waits on the host.
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "tnb_stages.cuh"

namespace tnb {

// ---------------------------------------------------------------------------------------
// the persistent chain kernel: every stage of a recorded chain in one launch

constexpr int kFusedThreads = 256;
constexpr int kMaxStages = 24;
constexpr long long kBarrierCycles = 4000000000LL;  // ~2 s at the boost clock

// A stage is a recorded op's words; data-buffer words equal to kSlotX / kSlotY stand for
// the launch's input and output vectors.
constexpr int64_t kSlotX = 1, kSlotY = 2;

// recorded op codes
constexpr int32_t kOpGather = 1;
constexpr int32_t kOpGemm = 2;
constexpr int32_t kOpFused = 3;
constexpr int32_t kOpGatherProduct = 4;
constexpr int32_t kOpCluster = 5;
constexpr int32_t kOpGemmGatherA = 6;
constexpr int32_t kOpGatherDirect = 7;

struct FStage {
  int32_t code;
  int32_t kind;
  int64_t items;
  int64_t w[16];
};

struct FChain {
  int32_t n;
  int32_t pad;
  FStage st[kMaxStages];
};

// 32 x 32 tiles run as four independent 64-thread groups per CTA (one tile each, own
// named barrier); gathers, skinny tiles and 64 x 64 tiles use the whole CTA.  (Gathers
// and skinny tiles split into groups measured slower: more dependent load rounds per
// item at the same number of loads in flight.)
constexpr int kGroups = 4, kGroupThreads = kFusedThreads / kGroups;

union FusedSmem {
  GatherSmem gather;
  GemmSmem<64, 64> g64;
  GemmSmem<32, 32> g32[kGroups];
  SkinnySmem skinny;
};

// Grid-wide barrier on two counters (arrivals, generation), zero before the first launch.
// Every wait is bounded: past the limit the CTA reports TNB_ETIMEOUT and the kernel ends.
__device__ bool grid_barrier(unsigned int* bar) {
  __syncthreads();
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    volatile unsigned int* gen = bar + 1;
    const unsigned int g = *gen;
    __threadfence();
    bool ok = true;
    if (atomicAdd(bar, 1u) == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const long long t0 = clock64();
      while (*gen == g) {
        if (clock64() - t0 > kBarrierCycles) {
          ok = false;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_ok = ok;
    if (!ok) atomicCAS(&g_device_error, 0, TNB_ETIMEOUT);
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ double* slot(int64_t w, const double* x, double* y) {
  return w == kSlotX ? const_cast<double*>(x)
                     : w == kSlotY ? y : reinterpret_cast<double*>(static_cast<intptr_t>(w));
}

// Every stage of a chain in order, `sync()` between stages (false: give up).
template <class Sync>
__device__ __forceinline__ void run_chain(const FChain& ch, const double* x, double* y,
                                          Sync sync) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FusedSmem& sm = *reinterpret_cast<FusedSmem*>(smem_raw);
  const int grp = threadIdx.x / kGroupThreads, gtid = threadIdx.x % kGroupThreads;
  const GroupSync gsync{1 + grp, kGroupThreads};
  for (int s = 0; s < ch.n; ++s) {
    const FStage& st = ch.st[s];
    const int64_t* w = st.w;
    if (st.code == kOpGather) {
      const GatherArgs g{reinterpret_cast<const int64_t*>(w[0]), w[1],
                         reinterpret_cast<const int32_t*>(w[2]),
                         reinterpret_cast<const int64_t*>(w[4]),
                         reinterpret_cast<const double*>(w[5]),
                         reinterpret_cast<const int64_t*>(w[6]), w[7], slot(w[8], x, y), w[9],
                         slot(w[10], x, y), w[11], slot(w[12], x, y), w[13], slot(w[14], x, y),
                         w[15]};
      for (int64_t it = blockIdx.x; it < st.items; it += gridDim.x)
        gather_chunk<kFusedThreads, true>(g, it, sm.gather, threadIdx.x, CtaSync{});
    } else {
      const int64_t poff = gemm_work_parts_offset(w[13]);
      char* work = reinterpret_cast<char*>(static_cast<intptr_t>(w[11]));
      const GemmArgs g{reinterpret_cast<const int64_t*>(w[0]), w[1],
                       reinterpret_cast<const int32_t*>(w[2]), slot(w[5], x, y), w[6],
                       slot(w[7], x, y), w[8], slot(w[9], x, y), w[10],
                       reinterpret_cast<unsigned int*>(work), w[13],
                       w[12] > poff ? reinterpret_cast<double*>(work + poff) : nullptr,
                       w[12] > poff ? (w[12] - poff) / 8 : 0};
      if (st.kind == TNB_TILE_64) {
        for (int64_t it = blockIdx.x; it < st.items; it += gridDim.x)
          gemm_tile<64, 64, true>(g, it, sm.g64, threadIdx.x, CtaSync{});
      } else if (st.kind == TNB_TILE_32) {
        for (int64_t it = static_cast<int64_t>(blockIdx.x) * kGroups + grp; it < st.items;
             it += static_cast<int64_t>(gridDim.x) * kGroups)
          gemm_tile<32, 32, true>(g, it, sm.g32[grp], gtid, gsync);
      } else {
        for (int64_t it = blockIdx.x; it < st.items; it += gridDim.x)
          skinny_tile<kFusedThreads, true>(g, it, sm.skinny, threadIdx.x, CtaSync{});
      }
    }
    if (s + 1 < ch.n && !sync()) return;
  }
}

struct GridStageSync {
  unsigned int* bar;
  __device__ __forceinline__ bool operator()() const { return grid_barrier(bar); }
};

struct ClusterStageSync {
  __device__ __forceinline__ bool operator()() const {
    __threadfence();
    asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
    return true;
  }
};

__global__ void __launch_bounds__(kFusedThreads, 1)
chain_kernel(const __grid_constant__ FChain ch, const double* x, double* y, unsigned int* bar) {
  run_chain(ch, x, y, GridStageSync{bar});
}

// The same chain on the CTAs of one thread-block cluster, the stages separated by the
// cluster's hardware barrier: for chains whose every stage has only a few dozen work
// items (a matvec at a small bond), where a grid-wide barrier or a launch per stage costs
// more than the stage.  The fence orders this CTA's global writes before the arrival;
// the barrier's release / acquire semantics at cluster scope make them visible to the
// other CTAs, which read them through L2.  Every CTA passes every barrier (no CTA leaves
// the loop early), so the barrier cannot wait on an exited CTA.
__global__ void __launch_bounds__(kFusedThreads, 1)
chain_cluster_kernel(const __grid_constant__ FChain ch, const double* x, double* y) {
  run_chain(ch, x, y, ClusterStageSync{});
}

// CTAs of one cooperative chain launch on `device`: as many as can be resident (0 when
// the kernel cannot be configured).
int fused_grid(int device) {
  static PerDeviceInt cached;
  int current = -1;
  if (cudaGetDevice(&current) != cudaSuccess || current != device) {
    cudaGetLastError();
    return 0;
  }
  return cached.get([](int dev, int* v) {
    const size_t smem = sizeof(FusedSmem);
    cudaError_t e = cudaFuncSetAttribute(chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    int per_sm = 0, sms = 0;
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, chain_kernel, kFusedThreads, smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    *v = per_sm * sms;
    return e;
  });
}

}  // namespace tnb

struct tnb_seq {
  struct Op {
    int32_t code;
    int64_t w[20];
  };
  std::vector<Op> ops;
  std::vector<tnb::FChain> chains;  // the stages of this sequence's fused ops
};

namespace tnb {
namespace {


// word positions of the data buffers a replay may substitute
constexpr int kGatherBufs[] = {8, 10, 12, 14};  // src0, dst0, src1, dst1
constexpr int kGemmBufs[] = {5, 7, 9};          // a, b, c
constexpr int kGatherProductBufs[] = {11, 13, 15};  // a, b, dst
constexpr int kGemmGatherABufs[] = {9, 11, 13};     // src, b, c
constexpr int kGatherDirectBufs[] = {6, 8, 10, 12};  // src0, dst0, src1, dst1

inline void* as_ptr(int64_t w) { return reinterpret_cast<void*>(static_cast<intptr_t>(w)); }
inline int64_t as_word(const void* p) { return static_cast<int64_t>(reinterpret_cast<intptr_t>(p)); }

int64_t patched(int64_t w, int32_t n_patch, const void* const* from, void* const* to) {
  for (int32_t i = 0; i < n_patch; ++i)
    if (w == as_word(from[i])) return as_word(to[i]);
  return w;
}

int replay(const tnb_seq* s, int32_t n_patch, const void* const* from, void* const* to,
           cudaStream_t stream) {
  for (const auto& op : s->ops) {
    int64_t w[20];
    std::memcpy(w, op.w, sizeof(w));
    int rc = TNB_EINVAL;
    if (op.code == kOpGather) {
      for (int k : kGatherBufs) w[k] = patched(w[k], n_patch, from, to);
      rc = tnb_block_gather(
          static_cast<const int64_t*>(as_ptr(w[0])), w[1], static_cast<const int32_t*>(as_ptr(w[2])),
          w[3], static_cast<const int64_t*>(as_ptr(w[4])), static_cast<const double*>(as_ptr(w[5])),
          static_cast<const int64_t*>(as_ptr(w[6])), w[7], static_cast<const double*>(as_ptr(w[8])),
          w[9], static_cast<double*>(as_ptr(w[10])), w[11],
          static_cast<const double*>(as_ptr(w[12])), w[13], static_cast<double*>(as_ptr(w[14])),
          w[15], stream);
    } else if (op.code == kOpGemm) {
      for (int k : kGemmBufs) w[k] = patched(w[k], n_patch, from, to);
      rc = tnb_grouped_gemm_f64(
          static_cast<const int64_t*>(as_ptr(w[0])), w[1], static_cast<const int32_t*>(as_ptr(w[2])),
          w[3], static_cast<int32_t>(w[4]), static_cast<const double*>(as_ptr(w[5])), w[6],
          static_cast<const double*>(as_ptr(w[7])), w[8], static_cast<double*>(as_ptr(w[9])), w[10],
          as_ptr(w[11]), w[12], w[13], stream);
    } else if (op.code == kOpGatherProduct) {
      for (int k : kGatherProductBufs) w[k] = patched(w[k], n_patch, from, to);
      rc = tnb_block_gather_product(
          static_cast<const int64_t*>(as_ptr(w[0])), w[1], static_cast<const int32_t*>(as_ptr(w[2])),
          w[3], static_cast<const int64_t*>(as_ptr(w[4])), static_cast<const double*>(as_ptr(w[5])),
          static_cast<const int64_t*>(as_ptr(w[6])), static_cast<const int64_t*>(as_ptr(w[7])),
          w[8], static_cast<const int64_t*>(as_ptr(w[9])), w[10],
          static_cast<const double*>(as_ptr(w[11])), w[12],
          static_cast<const double*>(as_ptr(w[13])), w[14],
          static_cast<double*>(as_ptr(w[15])), w[16], stream);
    } else if (op.code == kOpGatherDirect) {
      for (int k : kGatherDirectBufs) w[k] = patched(w[k], n_patch, from, to);
      rc = tnb_block_gather_direct(
          static_cast<const int64_t*>(as_ptr(w[0])), w[1],
          static_cast<const int64_t*>(as_ptr(w[2])), static_cast<const double*>(as_ptr(w[3])),
          static_cast<const int64_t*>(as_ptr(w[4])), w[5],
          static_cast<const double*>(as_ptr(w[6])), w[7], static_cast<double*>(as_ptr(w[8])),
          w[9], static_cast<const double*>(as_ptr(w[10])), w[11],
          static_cast<double*>(as_ptr(w[12])), w[13], stream);
    } else if (op.code == kOpGemmGatherA) {
      for (int k : kGemmGatherABufs) w[k] = patched(w[k], n_patch, from, to);
      rc = tnb_grouped_gemm_gather_a(
          static_cast<const int64_t*>(as_ptr(w[0])), w[1], static_cast<const int32_t*>(as_ptr(w[2])),
          w[3], static_cast<const int32_t*>(as_ptr(w[4])), w[5],
          static_cast<const int32_t*>(as_ptr(w[6])), static_cast<const double*>(as_ptr(w[7])),
          w[8], static_cast<const double*>(as_ptr(w[9])), w[10],
          static_cast<const double*>(as_ptr(w[11])), w[12], static_cast<double*>(as_ptr(w[13])),
          w[14], stream);
    } else if (op.code == kOpFused) {
      // w[0] chain index, w[1] input, w[2] output, w[3] barrier counters, w[4] grid
      w[1] = patched(w[1], n_patch, from, to);
      w[2] = patched(w[2], n_patch, from, to);
      if (w[0] < 0 || w[0] >= static_cast<int64_t>(s->chains.size())) {
        set_error("tnb_seq_run: corrupt fused op");
      } else {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(static_cast<unsigned>(w[4]));
        cfg.blockDim = dim3(kFusedThreads);
        cfg.dynamicSmemBytes = sizeof(FusedSmem);
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const cudaError_t e = cudaLaunchKernelEx(
            &cfg, chain_kernel, s->chains[static_cast<size_t>(w[0])],
            static_cast<const double*>(as_ptr(w[1])), static_cast<double*>(as_ptr(w[2])),
            static_cast<unsigned int*>(as_ptr(w[3])));
        if (e != cudaSuccess) {
          set_error(std::string("tnb_seq_run: fused chain launch: ") + cudaGetErrorString(e));
          rc = TNB_ECUDA;
        } else {
          rc = check_launch("tnb_seq_run: fused chain");
        }
      }
    } else if (op.code == kOpCluster) {
      // w[0] chain index, w[1] input, w[2] output, w[4] cluster size (the whole grid)
      w[1] = patched(w[1], n_patch, from, to);
      w[2] = patched(w[2], n_patch, from, to);
      if (w[0] < 0 || w[0] >= static_cast<int64_t>(s->chains.size()) || w[4] < 1 || w[4] > 16) {
        set_error("tnb_seq_run: corrupt cluster op");
        rc = TNB_EINVAL;
      } else {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(static_cast<unsigned>(w[4]));
        cfg.blockDim = dim3(kFusedThreads);
        cfg.dynamicSmemBytes = sizeof(FusedSmem);
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = static_cast<unsigned>(w[4]);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        const cudaError_t e = cudaLaunchKernelEx(
            &cfg, chain_cluster_kernel, s->chains[static_cast<size_t>(w[0])],
            static_cast<const double*>(as_ptr(w[1])), static_cast<double*>(as_ptr(w[2])));
        if (e != cudaSuccess) {
          set_error(std::string("tnb_seq_run: cluster chain launch: ") + cudaGetErrorString(e));
          rc = TNB_ECUDA;
        } else {
          rc = check_launch("tnb_seq_run: cluster chain");
        }
      }
    } else {
      set_error("tnb_seq_run: corrupt sequence");
    }
    if (rc != TNB_OK) return rc;
  }
  return TNB_OK;
}

}  // namespace
}  // namespace tnb

extern "C" int tnb_seq_create(tnb_seq** out) {
  TNB_REQUIRE(out != nullptr, "tnb_seq_create: out is null");
  *out = new (std::nothrow) tnb_seq();
  TNB_REQUIRE(*out != nullptr, "tnb_seq_create: out of host memory");
  return TNB_OK;
}

extern "C" void tnb_seq_destroy(tnb_seq* s) { delete s; }

extern "C" int64_t tnb_seq_length(const tnb_seq* s) {
  return s ? static_cast<int64_t>(s->ops.size()) : -1;
}

extern "C" int tnb_seq_add_gather(tnb_seq* s, const int64_t* seg_table, int64_t n_seg,
                                  const int32_t* chunk_map, int64_t total_chunks,
                                  const int64_t* term_src, const double* term_coeff,
                                  const int64_t* term_ld, int64_t n_term, const double* src0,
                                  int64_t n_src0, double* dst0, int64_t n_dst0,
                                  const double* src1, int64_t n_src1, double* dst1,
                                  int64_t n_dst1) {
  TNB_REQUIRE(s != nullptr, "tnb_seq_add_gather: null sequence");
  TNB_REQUIRE(n_seg >= 0 && total_chunks >= 0 && n_term >= 0, "tnb_seq_add_gather: negative size");
  using tnb::as_word;
  tnb_seq::Op op{tnb::kOpGather,
                 {as_word(seg_table), n_seg, as_word(chunk_map), total_chunks, as_word(term_src),
                  as_word(term_coeff), as_word(term_ld), n_term, as_word(src0), n_src0,
                  as_word(dst0), n_dst0, as_word(src1), n_src1, as_word(dst1), n_dst1}};
  s->ops.push_back(op);
  return TNB_OK;
}

extern "C" int tnb_seq_add_gemm(tnb_seq* s, const int64_t* gemm_table, int64_t n_gemm,
                                const int32_t* tile_map, int64_t total_tiles, int32_t tile_kind,
                                const double* a, int64_t n_a, const double* b, int64_t n_b,
                                double* c, int64_t n_c, void* work, int64_t work_bytes,
                                int64_t n_counters) {
  TNB_REQUIRE(s != nullptr, "tnb_seq_add_gemm: null sequence");
  TNB_REQUIRE(n_gemm >= 0 && total_tiles >= 0, "tnb_seq_add_gemm: negative size");
  using tnb::as_word;
  tnb_seq::Op op{tnb::kOpGemm,
                 {as_word(gemm_table), n_gemm, as_word(tile_map), total_tiles, tile_kind,
                  as_word(a), n_a, as_word(b), n_b, as_word(c), n_c, as_word(work), work_bytes,
                  n_counters, 0, 0}};
  s->ops.push_back(op);
  return TNB_OK;
}

extern "C" int tnb_seq_add_gather_direct(tnb_seq* s, const int64_t* chunk_rows,
                                         int64_t total_chunks, const int64_t* term_src,
                                         const double* term_coeff, const int64_t* term_ld,
                                         int64_t n_term, const double* src0, int64_t n_src0,
                                         double* dst0, int64_t n_dst0, const double* src1,
                                         int64_t n_src1, double* dst1, int64_t n_dst1) {
  TNB_REQUIRE(s != nullptr, "tnb_seq_add_gather_direct: null sequence");
  TNB_REQUIRE(total_chunks >= 0 && n_term >= 0, "tnb_seq_add_gather_direct: negative size");
  using tnb::as_word;
  tnb_seq::Op op{tnb::kOpGatherDirect,
                 {as_word(chunk_rows), total_chunks, as_word(term_src), as_word(term_coeff),
                  as_word(term_ld), n_term, as_word(src0), n_src0, as_word(dst0), n_dst0,
                  as_word(src1), n_src1, as_word(dst1), n_dst1}};
  s->ops.push_back(op);
  return TNB_OK;
}

extern "C" int tnb_seq_add_gemm_gather_a(tnb_seq* s, const int64_t* gemm_table, int64_t n_gemm,
                                         const int32_t* tile_map, int64_t total_tiles,
                                         const int32_t* a_ptr, int64_t n_ptr,
                                         const int32_t* a_src, const double* a_cf,
                                         int64_t n_terms, const double* src, int64_t n_src,
                                         const double* b, int64_t n_b, double* c, int64_t n_c) {
  TNB_REQUIRE(s != nullptr, "tnb_seq_add_gemm_gather_a: null sequence");
  TNB_REQUIRE(n_gemm >= 0 && total_tiles >= 0 && n_ptr >= 0 && n_terms >= 0,
              "tnb_seq_add_gemm_gather_a: negative size");
  using tnb::as_word;
  tnb_seq::Op op{tnb::kOpGemmGatherA,
                 {as_word(gemm_table), n_gemm, as_word(tile_map), total_tiles, as_word(a_ptr),
                  n_ptr, as_word(a_src), as_word(a_cf), n_terms, as_word(src), n_src,
                  as_word(b), n_b, as_word(c), n_c, 0}};
  s->ops.push_back(op);
  return TNB_OK;
}

extern "C" int tnb_seq_add_gather_product(tnb_seq* s, const int64_t* seg_table, int64_t n_seg,
                                          const int32_t* chunk_map, int64_t total_chunks,
                                          const int64_t* term_src, const double* term_coeff,
                                          const int64_t* term_ld, const int64_t* term_prod,
                                          int64_t n_term, const int64_t* prod_table,
                                          int64_t n_prod, const double* a, int64_t n_a,
                                          const double* b, int64_t n_b, double* dst,
                                          int64_t n_dst) {
  TNB_REQUIRE(s != nullptr, "tnb_seq_add_gather_product: null sequence");
  TNB_REQUIRE(n_seg >= 0 && total_chunks >= 0 && n_term >= 0 && n_prod >= 0,
              "tnb_seq_add_gather_product: negative size");
  using tnb::as_word;
  tnb_seq::Op op{tnb::kOpGatherProduct,
                 {as_word(seg_table), n_seg, as_word(chunk_map), total_chunks, as_word(term_src),
                  as_word(term_coeff), as_word(term_ld), as_word(term_prod), n_term,
                  as_word(prod_table), n_prod, as_word(a), n_a, as_word(b), n_b,
                  as_word(dst), n_dst, 0, 0, 0}};
  s->ops.push_back(op);
  return TNB_OK;
}

extern "C" int tnb_seq_append(tnb_seq* dst, const tnb_seq* src) {
  TNB_REQUIRE(dst != nullptr && src != nullptr, "tnb_seq_append: null sequence");
  TNB_REQUIRE(dst != src, "tnb_seq_append: a sequence cannot append itself");
  const int64_t base = static_cast<int64_t>(dst->chains.size());
  dst->chains.insert(dst->chains.end(), src->chains.begin(), src->chains.end());
  for (auto op : src->ops) {
    if (op.code == tnb::kOpFused || op.code == tnb::kOpCluster)
      op.w[0] += base;  // the copied chain's new index
    dst->ops.push_back(op);
  }
  return TNB_OK;
}

namespace tnb {
// The stages of `src` as a chain for the one-launch kernels; the slots' words become
// kSlotX / kSlotY so a replay can patch them.
static int build_chain(const tnb_seq* src, int64_t xw, int64_t yw, FChain& ch, const char* who) {
  if (src->ops.empty() || src->ops.size() > static_cast<size_t>(kMaxStages)) {
    set_error(std::string(who) + ": empty sequence or more stages than one launch holds");
    return TNB_EINVAL;
  }
  ch = FChain{};
  ch.n = static_cast<int32_t>(src->ops.size());
  for (size_t i = 0; i < src->ops.size(); ++i) {
    const auto& op = src->ops[i];
    FStage& st = ch.st[i];
    if (op.code != kOpGather && op.code != kOpGemm) {
      set_error(std::string(who) + ": only gathers and grouped GEMMs fuse (not product-source "
                "gathers or fused ops)");
      return TNB_EINVAL;
    }
    std::memcpy(st.w, op.w, sizeof(st.w));
    st.code = op.code;
    if (op.code == kOpGather) {
      st.kind = 0;
      st.items = op.w[3];  // chunks
      for (int k : kGatherBufs) st.w[k] = st.w[k] == xw ? kSlotX : st.w[k] == yw ? kSlotY : st.w[k];
    } else {
      st.kind = static_cast<int32_t>(op.w[4]);
      if (st.kind != TNB_TILE_64 && st.kind != TNB_TILE_32 && st.kind != TNB_TILE_SKINNY) {
        set_error(std::string(who) + ": only 64, 32 and skinny GEMM stages fuse");
        return TNB_EINVAL;
      }
      st.items = op.w[3];  // tiles (a 32 x 32 tile goes to one of four groups of a CTA)
      for (int k : kGemmBufs) st.w[k] = st.w[k] == xw ? kSlotX : st.w[k] == yw ? kSlotY : st.w[k];
    }
  }
  return TNB_OK;
}

// Largest cluster (16, 8, 4, 2 or 1 CTAs, at most `want`) of the cluster chain kernel
// that can be resident on the current device (0 if none); computed once per device.
static int cluster_size_for(int want) {
  static PerDeviceInt cached;
  const int best = cached.get([](int, int* v) {
    cudaError_t e = cudaFuncSetAttribute(chain_cluster_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(sizeof(FusedSmem)));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(chain_cluster_kernel,
                               cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    *v = 0;
    for (int c = 16; c >= 1 && *v == 0; c >>= 1) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(c);
      cfg.blockDim = dim3(kFusedThreads);
      cfg.dynamicSmemBytes = sizeof(FusedSmem);
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = c;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int clusters = 0;
      if (cudaOccupancyMaxActiveClusters(&clusters, chain_cluster_kernel, &cfg) == cudaSuccess &&
          clusters > 0)
        *v = c;
      else
        cudaGetLastError();
    }
    return *v > 0 ? cudaSuccess : cudaErrorInvalidConfiguration;
  });
  int c = best;
  while (c > want) c >>= 1;
  return c;
}
}  // namespace tnb

extern "C" int tnb_seq_fuse(const tnb_seq* src, const void* x_slot, const void* y_slot,
                            void* barrier, tnb_seq* dst) {
  TNB_REQUIRE(src != nullptr && dst != nullptr && src != dst, "tnb_seq_fuse: bad sequences");
  TNB_REQUIRE(x_slot != nullptr && y_slot != nullptr && barrier != nullptr,
              "tnb_seq_fuse: null slot or barrier");
  const int64_t xw = tnb::as_word(x_slot), yw = tnb::as_word(y_slot);
  tnb::FChain ch;
  if (int rc = tnb::build_chain(src, xw, yw, ch, "tnb_seq_fuse")) return rc;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    tnb::set_error("tnb_seq_fuse: no current device");
    return TNB_ECUDA;
  }
  const int grid = tnb::fused_grid(device);
  if (grid <= 0) {
    tnb::set_error("tnb_seq_fuse: the chain kernel cannot be resident");
    return TNB_ECUDA;
  }
  dst->chains.push_back(ch);
  tnb_seq::Op op{tnb::kOpFused,
                 {static_cast<int64_t>(dst->chains.size() - 1), xw, yw, tnb::as_word(barrier),
                  grid, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}};
  dst->ops.push_back(op);
  return TNB_OK;
}

extern "C" int tnb_seq_fuse_cluster(const tnb_seq* src, const void* x_slot, const void* y_slot,
                                    int32_t max_ctas, int32_t* ctas, tnb_seq* dst) {
  TNB_REQUIRE(src != nullptr && dst != nullptr && src != dst,
              "tnb_seq_fuse_cluster: bad sequences");
  TNB_REQUIRE(x_slot != nullptr && y_slot != nullptr, "tnb_seq_fuse_cluster: null slot");
  TNB_REQUIRE(max_ctas >= 1 && max_ctas <= 16, "tnb_seq_fuse_cluster: max_ctas must be 1..16");
  const int64_t xw = tnb::as_word(x_slot), yw = tnb::as_word(y_slot);
  tnb::FChain ch;
  if (int rc = tnb::build_chain(src, xw, yw, ch, "tnb_seq_fuse_cluster")) return rc;
  const int c = tnb::cluster_size_for(max_ctas);
  if (c <= 0) {
    tnb::set_error("tnb_seq_fuse_cluster: no cluster of the chain kernel can be resident");
    return TNB_ECUDA;
  }
  if (ctas) *ctas = c;
  dst->chains.push_back(ch);
  tnb_seq::Op op{tnb::kOpCluster,
                 {static_cast<int64_t>(dst->chains.size() - 1), xw, yw, 0, c, 0, 0, 0, 0, 0,
                  0, 0, 0, 0, 0, 0}};
  dst->ops.push_back(op);
  return TNB_OK;
}

extern "C" int tnb_seq_run(const tnb_seq* s, int32_t n_patch, const void* const* from,
                           void* const* to, void* stream) {
  TNB_REQUIRE(s != nullptr, "tnb_seq_run: null sequence");
  TNB_REQUIRE(n_patch >= 0 && (n_patch == 0 || (from && to)), "tnb_seq_run: bad patch list");
  return tnb::replay(s, n_patch, from, to, tnb::as_stream(stream));
}

#define TNB_TRY(expr)            \
  do {                           \
    const int rc_ = (expr);      \
    if (rc_ != TNB_OK) return rc_; \
  } while (0)

extern "C" int tnb_lanczos_solve(const tnb_seq* matvec, const void* x_slot, const void* y_slot,
                                 int64_t n, int32_t ncv, double tol, int32_t reorth,
                                 const double* x0, double* v, int64_t ldv, double* w,
                                 double* state, double* scal, const double* const* vptrs,
                                 double* gs, const int64_t* run_start, const double* run_w,
                                 int64_t n_runs, void* dot_work, void* multi_work,
                                 void* stream) {
  TNB_REQUIRE(matvec != nullptr, "tnb_lanczos_solve: null matvec sequence");
  TNB_REQUIRE(n > 0 && ncv > 0 && ldv >= n, "tnb_lanczos_solve: bad sizes");
  TNB_REQUIRE(x0 && v && w && state && scal && run_start && run_w && dot_work,
              "tnb_lanczos_solve: null buffer");
  TNB_REQUIRE(!reorth || (vptrs && gs && multi_work), "tnb_lanczos_solve: reorth buffers");
  cudaStream_t s = tnb::as_stream(stream);
  cudaError_t e = cudaMemsetAsync(state, 0, sizeof(double) * (3 * ncv + 2), s);
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_lanczos_solve: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  // v_0 = x0 / ||x0||
  TNB_TRY(tnb_weighted_dot(x0, x0, n, run_start, run_w, n_runs, dot_work, scal, stream));
  TNB_TRY(tnb_scale_rsqrt(n, scal, x0, v, stream));
  const void* from[2] = {x_slot, y_slot};
  // a vector one CTA can carry takes each step's five vector launches as one
  const bool one_cta = !reorth && n <= tnb_lanczos_step_max_n();
  for (int32_t j = 0; j < ncv; ++j) {
    double* vj = v + static_cast<int64_t>(j) * ldv;
    void* to[2] = {vj, w};
    TNB_TRY(tnb::replay(matvec, 2, from, to, s));
    if (one_cta) {
      TNB_TRY(tnb_lanczos_step(n, w, vj, j ? vj - ldv : nullptr, vj + ldv, state, j, ncv, tol,
                               run_start, run_w, n_runs, stream));
      continue;
    }
    TNB_TRY(tnb_weighted_dot(vj, w, n, run_start, run_w, n_runs, dot_work, state + j, stream));
    TNB_TRY(tnb_lanczos_update(n, w, vj, j ? vj - ldv : nullptr, state, j, ncv, stream));
    if (reorth) {
      for (int pass = 0; pass < 2; ++pass) {  // classical Gram-Schmidt, twice
        TNB_TRY(tnb_multi_dot(n, j + 1, vptrs, w, run_start, run_w, n_runs, multi_work, gs,
                              stream));
        TNB_TRY(tnb_lanczos_reorth(n, j + 1, gs, vptrs, w, state, ncv, stream));
      }
    }
    TNB_TRY(tnb_weighted_dot(w, w, n, run_start, run_w, n_runs, dot_work,
                             state + 2 * ncv + j, stream));
    TNB_TRY(tnb_lanczos_next(n, w, vj + ldv, state, j, ncv, tol, stream));
  }
  return TNB_OK;
}

extern "C" int tnb_lanczos_ritz(const tnb_seq* correct, const void* x_slot, const void* y_slot,
                                int64_t n, int32_t ncv, const double* coef,
                                const double* const* vptrs, double* out, double* w2,
                                double* scal, const int64_t* run_start, const double* run_w,
                                int64_t n_runs, void* dot_work, void* stream) {
  TNB_REQUIRE(n > 0 && ncv > 0, "tnb_lanczos_ritz: bad sizes");
  TNB_REQUIRE(coef && vptrs && out && scal && run_start && run_w && dot_work,
              "tnb_lanczos_ritz: null buffer");
  TNB_REQUIRE(!correct || w2, "tnb_lanczos_ritz: the correction needs w2");
  TNB_TRY(tnb_lincomb(n, ncv, coef, vptrs, out, stream));
  TNB_TRY(tnb_weighted_dot(out, out, n, run_start, run_w, n_runs, dot_work, scal, stream));
  TNB_TRY(tnb_scale_rsqrt(n, scal, out, out, stream));
  if (correct) {
    const void* from[2] = {x_slot, y_slot};
    void* to[2] = {out, w2};
    TNB_TRY(tnb::replay(correct, 2, from, to, tnb::as_stream(stream)));
    TNB_TRY(tnb_weighted_dot(out, w2, n, run_start, run_w, n_runs, dot_work, scal + 1, stream));
  }
  return TNB_OK;
}
