/*
 * tenet_b200.h -- C ABI of the B200 block-sparse symmetric-tensor engine.
 *
 * The reference (TeNeT-py) is pure Python: every block operation is an autoray
 * dispatch `ar.do(name, block, ...)` inside a per-block loop.  This library replaces
 * those loops with sm_100a kernels driven by flat descriptor tables that the Python
 * host planner builds once per tensor structure.  A maintainer binds it from Python
 * with ctypes; no torch type crosses this boundary.
 *
 * Conventions for every entry point
 *   - All pointers are DEVICE pointers to caller-owned memory unless stated; the
 *     library borrows them for the duration of the stream-ordered call only.
 *   - `stream` is a cudaStream_t passed as void*; 0 is the legacy default stream.
 *   - Return value: 0 on success, a nonzero TNB_E* code otherwise.  The message of
 *     the last failure on the calling host thread is tnb_last_error().  Nothing is
 *     launched when argument validation fails, so a refusal moves no data -- the
 *     reference's "refuse before any block moves" rule (ops/contraction.py:35-39).
 *   - Kernels bounds-check every table-driven access against the buffer lengths
 *     they are given.  A violation skips the access and raises a sticky device
 *     error word (never a trap); tnb_device_error() reads and clears it.
 *   - FP64 throughout the plain form.  Calls are thread-compatible: one stream per
 *     caller.  The only global state is the sticky device error word.
 */
#ifndef TENET_B200_H
#define TENET_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TNB_OK 0
#define TNB_EINVAL 1   /* bad argument (null pointer, negative size, bad table)   */
#define TNB_ECUDA 2    /* a CUDA runtime call failed                               */
#define TNB_EBOUNDS 3  /* a kernel saw an out-of-range table entry                 */
#define TNB_ETIMEOUT 4 /* a kernel gave up a bounded wait (tensor-core completion)  */

/* Maximum tensor rank a gather segment may carry. */
#define TNB_MAX_RANK 8

/*
 * Gather segment descriptor: one row of 40 int64 per destination block region.
 *
 *   [0]  dst_off       element offset of the region in its destination buffer
 *   [1]  size          number of elements (product of dims), < 2^31
 *   [2]  rank          number of dims used, 1..TNB_MAX_RANK
 *   [3]  t_begin       first term index (into term_src / term_coeff / term_ld)
 *   [4]  t_end         one past the last term index (t_end == t_begin: write zeros)
 *   [5]  buf           0 or 1: which (src, dst) buffer pair the segment uses
 *   [6]  chunk_begin   prefix sum of ceil(size / chunk) over earlier rows
 *   [7]  chunk         elements per work chunk of this row: 256, 512, 768 or 1024
 *                      (0 means TNB_GATHER_CHUNK); the host picks small chunks for small
 *                      tables (more CTAs on latency-bound work), large ones for big tables
 *   [8..15]  dims        iteration extents, outermost first
 *   [16..23] dst_stride  element stride of each dim in the destination
 *   [24..31] src_rstride source stride of each dim, in units of the term's ld
 *   [32..39] src_cstride source stride of each dim, in elements
 *
 * A source that is a plain block in an arena has src_rstride = 0; a source that is a
 * window of a coupled-sector matrix splits its strides into a row part (multiplied by
 * that matrix's leading dimension, which differs per term when the terms of one
 * destination come from different coupled sectors) and a column part.  For an element
 * with multi-index J, with R = sum_k J_k src_rstride_k and C = sum_k J_k src_cstride_k:
 *   dst[buf][dst_off + sum_k J_k dst_stride_k] =
 *       sum_{t in [t_begin, t_end)} term_coeff[t] * src[buf][term_src[t] + term_ld[t] * R + C]
 */
#define TNB_SEG_WIDTH 40
#define TNB_GATHER_CHUNK 1024

/*
 * Block gather-permute-scale-accumulate.  Replaces the per-term execution loops of
 *   transpose    ops/permutation.py:254-272   (blocks[dst] += c * transpose(blocks[src]))
 *   bend         ops/repartition.py:224-248
 *   repartition  ops/repartition.py:458-476
 * and, because a destination may be a strided window of a coupled-sector matrix, the
 * block <-> matrix lowering of
 *   to_matrices   map_view.py:238-279  (transpose + reshape + concatenate)
 *   from_matrices map_view.py:282-335  (slice + reshape + transpose)
 * Rows must be sorted by chunk_begin; total_chunks is the sum of all rows' chunks and
 * chunk_map[k] (int32, length total_chunks) is the row that chunk k belongs to.
 * Every destination element must belong to exactly one row (rows never overlap).
 */
int tnb_block_gather(const int64_t* seg_table, int64_t n_seg, const int32_t* chunk_map,
                     int64_t total_chunks,
                     const int64_t* term_src, const double* term_coeff,
                     const int64_t* term_ld, int64_t n_term,
                     const double* src0, int64_t n_src0, double* dst0, int64_t n_dst0,
                     const double* src1, int64_t n_src1, double* dst1, int64_t n_dst1,
                     void* stream);

/*
 * The same gather with its table as one row per chunk instead of rows + chunk map: row k
 * (TNB_CHUNK_ROW_WIDTH int64) is the segment row that chunk k belongs to (all 40 words,
 * word [6] still that segment's first chunk), then the segment's first term inline --
 * [40] term_src, [41] the bits of term_coeff, [42] term_ld -- a pad word, and [48 + d]
 * the division constant of extent d (mul = ceil(2^(31 + l) / dims[d]) with l =
 * ceil(log2 dims[d]) in the low 32 bits, l - 1 above them; 0 for an extent of 1), with
 * which element indices are split by a multiply and a shift (a constant without the
 * needed property falls back to division).  Every segment must have rank <= 4 (a
 * higher rank raises the bounds error; tnb_block_gather takes any).  A chunk of a
 * one-term segment (every segment of a U(1) / Z2 / fZ2 map) then reads its whole table in
 * one round of loads instead of three dependent ones (chunk map, row, terms), which is
 * what bounds many-wave gathers; segments with more terms read them from the term arrays
 * as tnb_block_gather does.  Same arithmetic and results, bit for bit.  No counterpart
 * in the reference (a table layout).
 */
#define TNB_CHUNK_ROW_WIDTH 56
int tnb_block_gather_direct(const int64_t* chunk_rows, int64_t total_chunks,
                            const int64_t* term_src, const double* term_coeff,
                            const int64_t* term_ld, int64_t n_term,
                            const double* src0, int64_t n_src0, double* dst0, int64_t n_dst0,
                            const double* src1, int64_t n_src1, double* dst1, int64_t n_dst1,
                            void* stream);

/*
 * Block gather whose source is a product with a short K, never materialised: the source
 * is C = A * B over the grouped-GEMM table prod_table (n_prod rows in the TNB_GEMM_WIDTH
 * layout below, K at most 4).  The segment rows are those of tnb_block_gather, with one
 * buffer pair (buf = 0); the terms address C by row and column instead of by offset:
 * term t of an element with row and column sums R and C (as above) reads
 *   C[m, n] = sum_{k < K} A[a_off + m * lda + k] * B[b_off + k * ldb + n],
 *   m = term_src[t] + R,  n = term_ld[t] + C,
 * of product row term_prod[t].  The product is computed where the gather reads it, with
 * the FMA chain of the FP64 GEMM kernels (from zero, k ascending), so the result is
 * bit-identical to tnb_grouped_gemm_f64 (any FP64 kind, no split-K) into a buffer
 * followed by tnb_block_gather over it -- one launch and one round trip of C fewer.  An
 * element outside its row's M x N block, or an operand access outside A or B, raises
 * the bounds error and reads 0.  No counterpart in the reference: its MPO links are a
 * matmul then a repartition (ops/map.py:155-172, ops/repartition.py:458-476).
 */
int tnb_block_gather_product(const int64_t* seg_table, int64_t n_seg,
                             const int32_t* chunk_map, int64_t total_chunks,
                             const int64_t* term_src, const double* term_coeff,
                             const int64_t* term_ld, const int64_t* term_prod, int64_t n_term,
                             const int64_t* prod_table, int64_t n_prod, const double* a,
                             int64_t n_a, const double* b, int64_t n_b, double* dst,
                             int64_t n_dst, void* stream);

/*
 * Grouped GEMM descriptor: one row of 16 int64 per product C = A * B (row-major).
 *
 *   [0] M  [1] N  [2] K  [3] a_off  [4] lda  [5] b_off  [6] ldb  [7] c_off  [8] ldc
 *   [9] tile_begin   prefix sum of tiles over earlier rows
 *   [10] tiles_n     number of tile columns (ceil(N / tile width); 1 for TNB_TILE_SKINNY)
 *   [11] tiles       number of tiles of this row (output tiles x splits)
 *   [12] splits      K splits per output tile (0 or 1: none); tiled kinds only
 *   [13] ksplit      K extent of one split, a multiple of 16
 *   [14] part_off    offset (in doubles) of this row's partial tiles in the work buffer
 *   [15] cnt_off     index of this row's first tile counter in the work buffer
 *
 * Split-K is deterministic: each split parks its partial tile, and the last of a tile's
 * splits to finish sums all of them in split order.  The work buffer holds n_counters
 * uint32 counters (padded to 256 bytes), then the partial tiles; its counters must be
 * zero before the first call (a fresh cudaMemset) and every call leaves them zero.
 * A table without splits may pass work = NULL, work_bytes = 0, n_counters = 0.
 *
 * K == 0 writes zeros (a coupled sector carried by one operand only).  All rows of one
 * launch use one tile kind:
 *   TNB_TILE_64      64 x 64 output tiles (tiles = ceil(M/64) * ceil(N/64))
 *   TNB_TILE_32      32 x 32 output tiles, for compositions too small to fill the GPU
 *   TNB_TILE_SKINNY  256 output rows per tile (tiles = ceil(M/256)); needs N, K <= 16
 *   TNB_TILE_WIDE    256 output columns per tile (tiles = ceil(N/256)); needs M, K <= 16
 *   TNB_TILE_TC_TF32    128 x 128 tiles on the tcgen05 tensor cores, operands rounded to
 *                       TF32, FP32 accumulation (tiles = ceil(M/128) * ceil(N/128))
 *   TNB_TILE_TC_3XBF16  same tiles, operands split into BF16 hi + lo pairs and the product
 *                       taken as hi.hi + hi.lo + lo.hi, FP32 accumulation
 * The tensor-core kinds read and write FP64 like the others; only the arithmetic inside
 * is reduced, and they take no split-K.  They pack each operand once into 16 KB slabs
 * (one 128-row x 32-K slab of A, or of B transposed, per slab) in the work buffer, so for
 * them columns [12] and [13] are the row's first A slab and first B slab (rows in slab
 * order, A slabs of a row m-tile-major then K), n_counters = A slabs | (B slabs << 32),
 * and work_bytes >= 16384 * (A slabs + B slabs); the work buffer needs no zeroing.
 */
#define TNB_GEMM_WIDTH 16
#define TNB_TILE_64 0
#define TNB_TILE_32 1
#define TNB_TILE_SKINNY 2
#define TNB_TILE_TC_TF32 3
#define TNB_TILE_TC_3XBF16 4
#define TNB_TILE_WIDE 5

/*
 * Grouped FP64 GEMM over uneven coupled sectors, one launch for every sector.
 * Replaces compose's per-sector loop ops/map.py:155-172 (`ar.do("matmul", ...)` per
 * coupled sector, zeros for a sector one operand lacks).  Rows sorted by tile_begin;
 * tile_map[k] (int32, length total_tiles) is the row that tile k belongs to.
 */
int tnb_grouped_gemm_f64(const int64_t* gemm_table, int64_t n_gemm, const int32_t* tile_map,
                         int64_t total_tiles, int32_t tile_kind, const double* a, int64_t n_a,
                         const double* b, int64_t n_b, double* c, int64_t n_c, void* work,
                         int64_t work_bytes, int64_t n_counters, void* stream);

/*
 * The FP64 tile kinds (TNB_TILE_64 / 32 / SKINNY / WIDE) of tnb_grouped_gemm_f64 with the
 * table as one TNB_GEMM_WIDTH row per tile -- row t is the row that tile t belongs to,
 * word [9] still that row's first tile -- instead of rows + tile map: a tile reads its row
 * in one load instead of two dependent ones.  Same arithmetic, split-K and work buffer, bit
 * for bit.  No counterpart in the reference (a table layout).
 */
int tnb_grouped_gemm_f64_rows(const int64_t* tile_rows, int64_t total_tiles, int32_t tile_kind,
                              const double* a, int64_t n_a, const double* b, int64_t n_b,
                              double* c, int64_t n_c, void* work, int64_t work_bytes,
                              int64_t n_counters, void* stream);

/*
 * A grouped FP64 GEMM whose A operand is a gather evaluated where it is read: the
 * to_matrices / repartition of the left operand (map_view.py:238-279,
 * ops/repartition.py:458-476) and compose's per-sector matmul (ops/map.py:155-172) in
 * one launch.  The table rows are TNB_GEMM_WIDTH rows of TNB_TILE_32 shape without
 * split-K (columns 12..15 zero), K <= 128, lda == K; a_off indexes the packed A, whose
 * element e is sum over t in [a_ptr[e], a_ptr[e+1]) of a_cf[t] * src[a_src[t]], summed
 * from zero in that order (a gather's own arithmetic).  n_ptr = packed A elements + 1.
 */
int tnb_grouped_gemm_gather_a(const int64_t* gemm_table, int64_t n_gemm, const int32_t* tile_map,
                              int64_t total_tiles, const int32_t* a_ptr, int64_t n_ptr,
                              const int32_t* a_src, const double* a_cf, int64_t n_terms,
                              const double* src, int64_t n_src, const double* b, int64_t n_b,
                              double* c, int64_t n_c, void* stream);

/*
 * Weighted inner product  out[0] = sum_r run_w[r] * sum_{i in run r} x[i] * y[i].
 * Runs are contiguous element ranges [run_start[r], run_start[r+1]) of equal weight
 * (consecutive blocks with the same qdim of their coupled sector merged).  Replaces
 *   inner  ops/contraction.py:517-589  (sum_tau qdim(c_tau) <A_tau, B_tau>)
 *   norm   ops/basic.py:309            (sqrt of inner(t, t))
 * `work` is caller-provided scratch of tnb_dot_work_bytes(n) bytes whose leading
 * counter word must be zero before the first call (a fresh cudaMemset); every call
 * leaves it zero again.  The reduction order is fixed, so results are deterministic.
 */
int64_t tnb_dot_work_bytes(int64_t n);
int tnb_weighted_dot(const double* x, const double* y, int64_t n,
                     const int64_t* run_start, const double* run_w, int64_t n_runs,
                     void* work, double* out, void* stream);

/*
 * Allocation-free weighted dot: the same result as tnb_weighted_dot (up to the order of
 * the partial sums), with no caller scratch.  No counterpart in the reference: it exists
 * for callers that cannot allocate device memory -- code being captured into a CUDA
 * graph under the global capture mode, where cudaMalloc is an error; a serving loop that
 * admits work against a fixed HBM budget and must not grow its footprint once a request
 * runs; a foreign-language host that holds only borrowed buffers and no allocator.
 *
 * Its scratch is a file-scope device array of 8448 bytes (a counter plus 1024 FP64
 * partials) that every GPU loading the library holds until exit, so n is limited to
 * TNB_DOT_NOALLOC_MAX_N = 2,097,152 elements; a larger n is refused with
 * TNB_EINVAL before anything runs.  The first call on a device looks up the array's
 * device address (set-up, once per device, with that device current): make that first
 * call before any stream capture.  cudaDeviceReset unloads the module and invalidates
 * the cached address: a call that then finds its launch refused looks the address up
 * again and retries once.  Each call zeroes the counter and overwrites the
 * partials; every call shares the one array, so calls that overlap on the GPU (two
 * streams at once) race -- serialise them.  No cudaMalloc, cudaFree or allocating
 * library routine is called.
 */
#define TNB_DOT_NOALLOC_MAX_N 2097152
int tnb_weighted_dot_noalloc(const double* x, const double* y, int64_t n,
                             const int64_t* run_start, const double* run_w, int64_t n_runs,
                             double* out, void* stream);

/*
 * dst[i] = src[i], i < n, by a kernel: either buffer may be pinned host memory (read or
 * written through its mapped device pointer), so a host caller's input and output move
 * inside the same stream -- or CUDA graph -- as the kernels around them, at about one
 * link latency per copy.  Pageable host memory is refused.  No counterpart in the
 * reference (its arrays live on one device already).
 */
int tnb_copy_f64(int64_t n, const double* src, double* dst, void* stream);

/*
 * *out = the address kernels use for `p`: `p` itself for device or managed memory, the
 * mapped device pointer for pinned host memory (so any kernel of this library may read
 * or write a pinned host buffer, e.g. the last gather of a matvec writing its result to
 * the host directly).  TNB_EINVAL for pageable host memory.
 */
int tnb_mapped_address(const void* p, void** out);

/*
 * out[i] = alpha * x[i] + beta * y[i], i < n.  `out` may alias `x` or `y`.
 * Replaces add / subtract / multiply / divide over aligned blocks
 * (ops/basic.py:81-236) and Lanczos' vector updates (network/dmrg.py:207-227).
 */
int tnb_axpby(int64_t n, double alpha, const double* x, double beta, const double* y,
              double* out, void* stream);

/*
 * Device-resident Lanczos (network/dmrg.py:106-227 without host round trips).  `state`
 * holds 3 ncv + 2 doubles: alpha[0, ncv), beta[ncv, 2 ncv), squared norms [2 ncv, 3 ncv),
 * the Krylov size m at [3 ncv] and a stopped flag at [3 ncv + 1], zeroed before step 0.
 * Step j of the three-term recurrence, with w = H v_j and alpha[j] = <v_j, w> already
 * written (tnb_weighted_dot into state + j):
 *   tnb_lanczos_update  w <- w - alpha_j v_j - beta_{j-1} v_{j-1}   (no-op once stopped)
 *   (tnb_weighted_dot of w with itself into state + 2 ncv + j)
 *   tnb_lanczos_next    beta_j = ||w||; stop when j + 1 == ncv or beta_j < tol (the
 *                       reference's happy breakdown); else v_{j+1} = w / beta_j, beta[j]
 *                       and m = j + 2 recorded; once stopped v_{j+1} = 0.
 * tnb_scale_rsqrt: out = x / sqrt(s2[0]) with s2 a device scalar (normalisation by a
 * device-side squared norm).
 */
int tnb_lanczos_update(int64_t n, double* w, const double* v, const double* vprev,
                       const double* state, int32_t j, int32_t ncv, void* stream);
int tnb_lanczos_next(int64_t n, const double* w, double* vnext, double* state, int32_t j,
                     int32_t ncv, double tol, void* stream);
int tnb_scale_rsqrt(int64_t n, const double* s2, const double* x, double* out, void* stream);

/*
 * The whole of step j after the matvec for a vector of n <= tnb_lanczos_step_max_n()
 * doubles, in one launch of one CTA: alpha_j = <v_j, w> into state + j, the update,
 * ||w||^2 into state + 2 ncv + j and the stop decision with v_{j+1} (vnext) -- what
 * tnb_weighted_dot, tnb_lanczos_update, tnb_weighted_dot and tnb_lanczos_next do in five
 * launches, with their arithmetic (for n <= 2048 the same bits).  Once `state` says the
 * recurrence stopped it only zeroes vnext.  tnb_lanczos_solve takes it for such vectors
 * when it does not reorthogonalise.
 */
int64_t tnb_lanczos_step_max_n(void);
int tnb_lanczos_step(int64_t n, double* w, const double* v, const double* vprev, double* vnext,
                     double* state, int32_t j, int32_t ncv, double tol, const int64_t* run_start,
                     const double* run_w, int64_t n_runs, void* stream);

/*
 * FP64 reorthogonalisation for the precision form (no counterpart in the reference,
 * whose Lanczos is not reorthogonalised): tnb_multi_dot writes out[j] = <vecs[j], x>
 * (qdim-weighted, runs as tnb_weighted_dot) for j < k in one pass with caller scratch of
 * tnb_multi_dot_work_bytes(n, k) bytes (counter zero before first use, left zero);
 * tnb_lanczos_reorth does w -= sum_j coeffs[j] vecs[j] (a no-op once `state` says the
 * recurrence stopped; state may be NULL).  vecs and coeffs are device arrays.
 */
int64_t tnb_multi_dot_work_bytes(int64_t n, int64_t k);
int tnb_multi_dot(int64_t n, int64_t k, const double* const* vecs, const double* x,
                  const int64_t* run_start, const double* run_w, int64_t n_runs, void* work,
                  double* out, void* stream);
int tnb_lanczos_reorth(int64_t n, int64_t k, const double* coeffs, const double* const* vecs,
                       double* w, const double* state, int32_t ncv, void* stream);

/*
 * out[i] = sum_j coeffs[j] * vecs[j][i] for j < k, i < n.  `vecs` is a DEVICE array of
 * k device pointers; `coeffs` a DEVICE array of k doubles.  The Lanczos Ritz-vector
 * recombination (network/dmrg.py:224-227) in one pass.
 */
int tnb_lincomb(int64_t n, int64_t k, const double* coeffs, const double* const* vecs,
                double* out, void* stream);

/*
 * Enable (1) or disable (0) programmatic dependent launch for the table-driven kernels
 * (tnb_block_gather, tnb_grouped_gemm_f64); returns the previous setting.  When enabled,
 * each such kernel lets the next kernel of the stream begin loading its own static
 * tables while it runs, and waits for the previous kernel's results before reading them;
 * results are identical either way.  Default: enabled.
 */
int tnb_set_pdl(int enabled);

/*
 * Recorded launch sequences (no counterpart in the reference, whose per-block loops run
 * in Python; this is the native replacement of the host loop around them).  A sequence
 * records tnb_block_gather / tnb_grouped_gemm_f64 launches -- tables, buffers, sizes --
 * and tnb_seq_run replays them in order on `stream`, first substituting every data
 * buffer pointer equal to from[i] by to[i] (HOST arrays of n_patch pointers; 0 = none).
 * A compiled matvec is recorded once on placeholder input/output buffers and replayed
 * on any vectors of the same sizes.  The sequence borrows every recorded pointer: the
 * caller keeps tables and buffers alive while it may run.  Replay returns the first
 * failing launch's status.  A sequence is not thread-safe; replays only read it.
 */
typedef struct tnb_seq tnb_seq;
int tnb_seq_create(tnb_seq** out);
void tnb_seq_destroy(tnb_seq* s);
int64_t tnb_seq_length(const tnb_seq* s);
int tnb_seq_add_gather(tnb_seq* s, const int64_t* seg_table, int64_t n_seg,
                       const int32_t* chunk_map, int64_t total_chunks, const int64_t* term_src,
                       const double* term_coeff, const int64_t* term_ld, int64_t n_term,
                       const double* src0, int64_t n_src0, double* dst0, int64_t n_dst0,
                       const double* src1, int64_t n_src1, double* dst1, int64_t n_dst1);
/* Records a tnb_block_gather_direct launch (the per-chunk-row table form). */
int tnb_seq_add_gather_direct(tnb_seq* s, const int64_t* chunk_rows, int64_t total_chunks,
                              const int64_t* term_src, const double* term_coeff,
                              const int64_t* term_ld, int64_t n_term, const double* src0,
                              int64_t n_src0, double* dst0, int64_t n_dst0, const double* src1,
                              int64_t n_src1, double* dst1, int64_t n_dst1);
int tnb_seq_add_gemm(tnb_seq* s, const int64_t* gemm_table, int64_t n_gemm,
                     const int32_t* tile_map, int64_t total_tiles, int32_t tile_kind,
                     const double* a, int64_t n_a, const double* b, int64_t n_b, double* c,
                     int64_t n_c, void* work, int64_t work_bytes, int64_t n_counters);
int tnb_seq_add_gather_product(tnb_seq* s, const int64_t* seg_table, int64_t n_seg,
                               const int32_t* chunk_map, int64_t total_chunks,
                               const int64_t* term_src, const double* term_coeff,
                               const int64_t* term_ld, const int64_t* term_prod,
                               int64_t n_term, const int64_t* prod_table, int64_t n_prod,
                               const double* a, int64_t n_a, const double* b, int64_t n_b,
                               double* dst, int64_t n_dst);
int tnb_seq_append(tnb_seq* dst, const tnb_seq* src);

/*
 * Fuse a recorded sequence of gathers and FP64 grouped GEMMs (kinds 64, 32, skinny; at
 * most 24 ops) into ONE launch appended to `dst`: a persistent cooperative kernel, as
 * many 256-thread CTAs as can be resident, that runs the stages in order with a
 * grid-wide barrier between them (each stage's tables and arithmetic are those of its
 * standalone kernel, so results are bit-identical).  Data-buffer pointers equal to
 * x_slot / y_slot become the launch's input / output, which tnb_seq_run's patch list
 * substitutes like any buffer.  `barrier` is 8 bytes of device memory, zero before the
 * first launch, owned by this fused op alone: two launches of it must not overlap.  Its
 * waits are bounded (about 2 s): past the limit the device error word reads
 * TNB_ETIMEOUT and the counters must be zeroed again.  Tensor-core stages are refused
 * (TNB_EINVAL).  Replaces no reference interface (the reference runs each block map and
 * composition as its own Python loop); it is the one-launch form of a compiled chain.
 */
int tnb_seq_add_gemm_gather_a(tnb_seq* s, const int64_t* gemm_table, int64_t n_gemm,
                              const int32_t* tile_map, int64_t total_tiles, const int32_t* a_ptr,
                              int64_t n_ptr, const int32_t* a_src, const double* a_cf,
                              int64_t n_terms, const double* src, int64_t n_src, const double* b,
                              int64_t n_b, double* c, int64_t n_c);
int tnb_seq_fuse(const tnb_seq* src, const void* x_slot, const void* y_slot, void* barrier,
                 tnb_seq* dst);

/*
 * The stages of `src` as one launch on a single thread-block cluster of up to `max_ctas`
 * (1..16) CTAs, the stages separated by the cluster's hardware barrier, appended to `dst`
 * as one op (*ctas = the cluster size used: the largest power of two <= max_ctas that
 * the device can make resident).  For chains whose stages each have a few dozen work
 * items -- a two-site matvec at a small bond -- where a launch per stage or a grid-wide
 * barrier costs more than the stage.  No counterpart in the reference (its matvec is a
 * Python loop of per-block calls); the stages are the same tables as the op-by-op
 * sequence, so the results are bit-identical.
 */
int tnb_seq_fuse_cluster(const tnb_seq* src, const void* x_slot, const void* y_slot,
                         int32_t max_ctas, int32_t* ctas, tnb_seq* dst);
int tnb_seq_run(const tnb_seq* s, int32_t n_patch, const void* const* from, void* const* to,
                void* stream);

/*
 * One whole Lanczos solve from one host call (replaces the loop of
 * network/dmrg.py:106-227): zero `state`, v_0 = x0/||x0||, then for j < ncv the matvec
 * sequence replayed with x_slot -> v_j and y_slot -> w, alpha_j, tnb_lanczos_update,
 * optional classical Gram-Schmidt twice against v_0..v_j (reorth != 0; vptrs = DEVICE
 * array of the ncv row pointers of v, gs = ncv doubles, multi_work of
 * tnb_multi_dot_work_bytes(n, ncv) bytes), ||w||^2 and tnb_lanczos_next.  `v` holds
 * ncv + 1 rows of stride ldv >= n; `scal` 2 doubles; dot_work tnb_dot_work_bytes(n).
 * The caller reads `state` (one synchronising copy), solves the tridiagonal, and calls
 * tnb_lanczos_ritz: out = normalised sum_j coef[j] v_j, and, when `correct` is given
 * (the FP64 sequence of the precision form), scal[1] = <out, H out> with H out in w2.
 */
int tnb_lanczos_solve(const tnb_seq* matvec, const void* x_slot, const void* y_slot, int64_t n,
                      int32_t ncv, double tol, int32_t reorth, const double* x0, double* v,
                      int64_t ldv, double* w, double* state, double* scal,
                      const double* const* vptrs, double* gs, const int64_t* run_start,
                      const double* run_w, int64_t n_runs, void* dot_work, void* multi_work,
                      void* stream);
int tnb_lanczos_ritz(const tnb_seq* correct, const void* x_slot, const void* y_slot, int64_t n,
                     int32_t ncv, const double* coef, const double* const* vptrs, double* out,
                     double* w2, double* scal, const int64_t* run_start, const double* run_w,
                     int64_t n_runs, void* dot_work, void* stream);

/*
 * Host-side planner kernels (no device; plain loops over host arrays).  They replace the
 * per-block loops of the table builder (the reference runs its block maps directly:
 * ops/permutation.py:254-272, ops/repartition.py:298-316).
 *
 * tnb_plan_gather_rows: one TNB_SEG_WIDTH row per destination block r < n_rows from its
 *   dims, destination strides, source row/column strides (n_rows x nd, row-major, the
 *   source's permuted to destination axis order), offset, size and term range: dims
 *   ordered by destination stride (descending; ties by source column, then row stride,
 *   stable), extent-1 dims dropped, dims contiguous in destination and source merged,
 *   a rank-1 unit row when nothing is left.  TNB_EINVAL when a row keeps more than
 *   TNB_MAX_RANK dims.
 * tnb_plan_gather_table: the whole gather table of a block map: terms (t_src, t_dst,
 *   t_coef; n_terms) over source blocks (n_src: offset, leading dimension, and nd row / column
 *   strides each) and destination blocks (n_dst: offset, nd strides, nd dims, size, keep
 *   flag), `perm` giving for each destination axis its source axis.  The terms of kept
 *   destination blocks, grouped by destination block in block order (their given order
 *   kept), become one row each per block (tnb_plan_gather_rows' rules, the first term's
 *   source strides permuted) and fill out_src / out_coef / out_ld (source offset,
 *   coefficient, leading dimension per term); every kept block without terms then gets a
 *   zero-writing row.  rows holds n_dst rows, the term outputs n_terms entries; counts[0]
 *   = rows written, counts[1] = terms written.  TNB_EINVAL on an out-of-range index or a
 *   row above TNB_MAX_RANK dims.
 * tnb_plan_compose: the sparse product of block maps a (n_a x 3: src, mid, coeff) and
 *   b (n_b x 3: mid, dst, coeff): each (src, dst) pair once, in order of first occurrence
 *   walking a in order and b's terms of each mid in their order, coefficients summed in
 *   that order from zero.  Writes at most `cap` rows to `out`; returns the row count, -1
 *   on a bad argument, -2 when `cap` is too small.
 */
int tnb_plan_gather_rows(int64_t n_rows, int32_t nd, const int64_t* dims, const int64_t* dstr,
                         const int64_t* rstr, const int64_t* cstr, const int64_t* d_off,
                         const int64_t* sizes, const int64_t* t_begin, const int64_t* t_end,
                         int64_t buf, int64_t* rows);
int tnb_plan_gather_table(int64_t n_terms, const int64_t* t_src, const int64_t* t_dst,
                          const double* t_coef, int64_t n_src, const int64_t* s_off,
                          const int64_t* s_ld, const int64_t* s_rs, const int64_t* s_cs,
                          int64_t n_dst, const int64_t* d_off, const int64_t* d_str,
                          const int64_t* d_shape, const int64_t* d_size, const uint8_t* keep,
                          int32_t nd, const int64_t* perm, int64_t buf, int64_t* rows,
                          int64_t* out_src, double* out_coef, int64_t* out_ld, int64_t* counts);
int64_t tnb_plan_compose(int64_t n_a, const double* a, int64_t n_b, const double* b, double* out,
                         int64_t cap);

/*
 * Blockwise SVD of the coupled-sector matrices of a lowered tensor.  Replaces the
 * reference's per-sector `ar.do("linalg.svd")` loop of svd_truncated
 * (ops/linalg.py:1593-1612).  One CTA per row of `rows` (8 int64 each):
 *   [0] m, [1] n         the sector matrix, row-major at a + a_off
 *   [2] a_off
 *   [3] u_off            U (m x k, row-major), k = min(m, n)
 *   [4] s_off            singular values (k), descending
 *   [5] vt_off           Vh (k x n, row-major)
 *   [6] w_off            -1: the working copy (max(m,n) k + k^2 + 2k doubles) lives in
 *                        `smem_doubles` of dynamic shared memory (at most
 *                        tnb_block_svd_smem_doubles()); else its offset in `work`
 *   [7] 0
 * One-sided Jacobi (rotations until every column pair is orthogonal to 1e-15 relative);
 * columns of exactly zero norm get an orthonormal completion.  info[row] = 0 on
 * convergence, the sweep count if the 64-sweep limit was reached, -1 on a bad row.
 */
int64_t tnb_block_svd_smem_doubles(void);
int tnb_block_svd(const int64_t* rows, int64_t n_rows, const double* a, int64_t n_a,
                  double* u, int64_t n_u, double* s, int64_t n_s, double* vt, int64_t n_vt,
                  double* work, int64_t n_work, int32_t* info, int64_t smem_doubles,
                  void* stream);

/*
 * The truncation decision on the device: _spectrum / _admissible / _decide of
 * ops/linalg.py:1079-1324 in one CTA.  sectors: n_sec rows of 4 int64 [count, s_off,
 * label, 0] in ascending label order, each a descending list of `count` singular values
 * at s + s_off; qdim: the sectors' quantum dimensions.  The global order is (-sigma,
 * sector, index); mode 0..5 = abs, rel, sum2, rsum2, sum1, rsum1 with `cutoff` (< 0: no
 * cutoff); max_bond (< 0: none) bounds sum qdim (budget 0) or the count (budget 1) of the
 * kept values, the walk stopping at the first overflow.  The sums run in the reference's
 * order.  Outputs: keep[sector] counts, the global order (sorted_s, sorted_c: sector
 * index), stats = {kept, dense dim, discarded weight, total weight, kept weight,
 * admissible, total count, 0}.
 */
int tnb_truncate_decide(const int64_t* sectors, const double* qdim, int64_t n_sec,
                        const double* s, int64_t n_s, double cutoff, int32_t mode,
                        double max_bond, int32_t budget, int64_t* keep, double* sorted_s,
                        int32_t* sorted_c, double* stats, void* stream);

/*
 * The kept prefixes into the truncated factors' packed coupled-sector matrices
 * (ops/linalg.py:1599-1612): rows of 12 int64 [m, n, k_full, k, u_off, s_off, vt_off,
 * pu_off, ps_off, pv_off, 0, 0] -> PU (m x k) = U[:, :k], PS (k x k) = diag(s[:k]) *
 * scale, PV (k x n) = Vh[:k, :].
 */
int tnb_svd_compact(const int64_t* rows, int64_t n_rows, const double* u, int64_t n_u,
                    const double* s, int64_t n_s, const double* vt, int64_t n_vt,
                    double scale, double* pu, int64_t n_pu, double* ps, int64_t n_ps,
                    double* pv, int64_t n_pv, void* stream);

/*
 * Blockwise LQ (replaces the per-sector QR loop of `lq`, ops/linalg.py:549-620, which
 * factors each coupled sector's B^T).  One CTA per sector; `rows` holds n_rows rows of 8
 * int64 [mb, nb, b_off, l_off, q_off, w_off, 0, 0]: B (mb x nb, row-major) at b + b_off is
 * factored as B^T = Q R by Householder reflections in LAPACK's convention (dgeqrf/dorgqr:
 * beta = -sign(alpha) |x|, tau = (beta - alpha) / beta, tau = 0 when nothing lies below
 * the diagonal), giving L = R^T (mb x k) at l + l_off and Q^T (k x nb) at q + q_off,
 * k = min(mb, nb), both row-major.  The work area (nb*mb + nb*k + 2k doubles) is dynamic
 * shared memory when w_off < 0 (smem_doubles <= tnb_block_svd_smem_doubles()), else
 * work + w_off.  Bounds are checked per row (TNB_EBOUNDS on the device word).
 */
int tnb_block_lq(const int64_t* rows, int64_t n_rows, const double* b, int64_t n_b,
                 double* l, int64_t n_l, double* q, int64_t n_q, double* work, int64_t n_work,
                 int64_t smem_doubles, void* stream);

/* Library version (major*10000 + minor*100 + patch). */
int tnb_version(void);

/* Message of the last failed call on this host thread ("" if none). */
const char* tnb_last_error(void);

/*
 * Read and clear the sticky device error word (0 = clean, else the TNB_E* code a
 * kernel raised).  Synchronises `stream`.
 */
int tnb_device_error(int* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* TENET_B200_H */
