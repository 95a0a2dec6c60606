// K4: blockwise SVD and the truncation decision on the device.
//
// The reference factorises each coupled-sector matrix of the lowered tensor with one
// `ar.do("linalg.svd")` call (ops/linalg.py:1593-1612), pulls every singular value to the
// host as a Python float, sorts the global spectrum by (-sigma, sector, index)
// (_spectrum, linalg.py:1079-1097) and walks it with the cutoff prefix and the dense
// budget (_admissible / _decide, linalg.py:1100-1324).  Here:
//
//   block_svd_kernel   one CTA per sector: one-sided Jacobi (Hestenes) on the taller
//                      orientation of the matrix, columns rotated in round-robin order,
//                      rotations accumulated into V; singular values are the final column
//                      norms, sorted descending; a column whose norm is exactly zero gets
//                      an orthonormal completion (so U and Vh stay isometries).  The
//                      working copy lives in shared memory when it fits, else in the
//                      caller's global work buffer.
//   decide_kernel      one CTA: the global order by rank (binary searches in the sorted
//                      per-sector lists), then the reference's sequential cutoff and
//                      budget walk in the same summation order.
//   svd_compact_kernel the kept prefixes of U, S (times the renormalisation) and Vh into
//                      the packed coupled-sector layouts of the truncated factors.
#include <cmath>
#include <string>

#include "tnb_common.cuh"

namespace tnb {

constexpr int kSvdThreads = 512;
constexpr int kSvdWarps = kSvdThreads / 32;
constexpr int kSvdMaxSweeps = 64;
constexpr double kSvdTol = 1e-15;  // rotate while |a_i . a_j| > tol * |a_i| |a_j|
constexpr int kSvdRow = 8;         // m, n, a_off, u_off, s_off, vt_off, w_off, pad
constexpr int kDecideThreads = 1024;
constexpr int kSectorRow = 4;      // count, s_off, label, pad (qdim in a double array)
constexpr int kCompactRow = 12;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Column pair of round-robin step `step` (0 <= step < cp - 1) and pair `k` (0 <= k <
// cp / 2) for an even column count cp: every pair of columns meets once per sweep.
__device__ __forceinline__ void rr_pair(int cp, int step, int k, int& i, int& j) {
  const int n1 = cp - 1;
  if (k == 0) {
    i = n1;
    j = step;
  } else {
    i = (step + k) % n1;
    j = (step - k + n1) % n1;
  }
  if (i > j) {
    const int t = i;
    i = j;
    j = t;
  }
}

// CTA-wide sum of one value per thread (every thread gets the result).
__device__ double cta_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < kSvdWarps; ++w) t += red[w];
  return t;
}

__global__ void __launch_bounds__(kSvdThreads)
block_svd_kernel(const int64_t* __restrict__ rows, int64_t n_rows, const double* __restrict__ a,
                 int64_t n_a, double* __restrict__ u, int64_t n_u, double* __restrict__ s,
                 int64_t n_s, double* __restrict__ vt, int64_t n_vt, double* __restrict__ work,
                 int64_t n_work, int32_t* __restrict__ info, int64_t smem_doubles) {
  extern __shared__ __align__(16) double svd_smem[];
  __shared__ double red[kSvdWarps];
  __shared__ int s_rotated;
  const int64_t b = blockIdx.x;
  if (b >= n_rows) return;
  const int64_t* row = rows + b * kSvdRow;
  const int64_t m = row[0], n = row[1], a_off = row[2], u_off = row[3], s_off = row[4],
                vt_off = row[5], w_off = row[6];
  const bool trans = m < n;
  const int64_t r = trans ? n : m, c = trans ? m : n;  // W = A or A^T: r x c, r >= c
  const bool ok = m >= 0 && n >= 0 && c <= 4096 && a_off >= 0 && a_off + m * n <= n_a &&
                  u_off >= 0 && u_off + m * c <= n_u && s_off >= 0 && s_off + c <= n_s &&
                  vt_off >= 0 && vt_off + c * n <= n_vt &&
                  (w_off >= 0 ? w_off + r * c + c * c + 2 * c <= n_work
                              : r * c + c * c + 2 * c <= smem_doubles);
  if (!ok) {
    if (threadIdx.x == 0) {
      raise_bounds();
      info[b] = -1;
    }
    return;
  }
  if (c == 0) {
    if (threadIdx.x == 0) info[b] = 0;
    return;
  }
  double* W = w_off >= 0 ? work + w_off : svd_smem;  // column j at W + j * r
  double* V = W + r * c;                               // column j at V + j * c
  double* sig = V + c * c;
  double* pos = sig + c;  // sorted position of column j (an integer, held as a double)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

  for (int64_t e = tid; e < r * c; e += kSvdThreads) {
    const int64_t j = e / r, i = e % r;
    W[e] = trans ? a[a_off + j * n + i] : a[a_off + i * n + j];
  }
  for (int64_t e = tid; e < c * c; e += kSvdThreads) V[e] = (e / c == e % c) ? 1.0 : 0.0;
  __syncthreads();

  const int cp = static_cast<int>(c + (c & 1));
  int sweep = 0;
  bool converged = c == 1;
  for (; sweep < kSvdMaxSweeps && !converged; ++sweep) {
    if (tid == 0) s_rotated = 0;
    __syncthreads();
    for (int step = 0; step < cp - 1; ++step) {
      for (int k = warp; k < cp / 2; k += kSvdWarps) {
        int i, j;
        rr_pair(cp, step, k, i, j);
        if (j >= c) continue;  // the padding column
        double* wi = W + static_cast<int64_t>(i) * r;
        double* wj = W + static_cast<int64_t>(j) * r;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int64_t q = lane; q < r; q += 32) {
          const double x = wi[q], y = wj[q];
          al = fma(x, x, al);
          be = fma(y, y, be);
          ga = fma(x, y, ga);
        }
        al = warp_sum(al);
        be = warp_sum(be);
        ga = warp_sum(ga);
        if (!(fabs(ga) > kSvdTol * sqrt(al) * sqrt(be)) || al == 0.0 || be == 0.0) continue;
        const double zeta = (be - al) / (2.0 * ga);
        const double t = fabs(zeta) > 1e150
                             ? 0.5 / zeta
                             : copysign(1.0, zeta) / (fabs(zeta) + sqrt(fma(zeta, zeta, 1.0)));
        const double cs = 1.0 / sqrt(fma(t, t, 1.0)), sn = cs * t;
        for (int64_t q = lane; q < r; q += 32) {
          const double x = wi[q], y = wj[q];
          wi[q] = cs * x - sn * y;
          wj[q] = sn * x + cs * y;
        }
        double* vi = V + static_cast<int64_t>(i) * c;
        double* vj = V + static_cast<int64_t>(j) * c;
        for (int64_t q = lane; q < c; q += 32) {
          const double x = vi[q], y = vj[q];
          vi[q] = cs * x - sn * y;
          vj[q] = sn * x + cs * y;
        }
        if (lane == 0) s_rotated = 1;
      }
      __syncthreads();
    }
    converged = s_rotated == 0;
    __syncthreads();
  }

  // singular values: the column norms
  for (int64_t j = warp; j < c; j += kSvdWarps) {
    const double* wj = W + j * r;
    double x = 0.0;
    for (int64_t q = lane; q < r; q += 32) x = fma(wj[q], wj[q], x);
    x = warp_sum(x);
    if (lane == 0) sig[j] = sqrt(x);
  }
  __syncthreads();
  // normalise the nonzero columns
  for (int64_t e = tid; e < r * c; e += kSvdThreads) {
    const double sj = sig[e / r];
    if (sj > 0.0) W[e] /= sj;
  }
  __syncthreads();

  // rank of each column in descending order (ties by column index), then the
  // completion of exactly-zero columns in that order: a unit vector orthogonalised
  // (twice) against every column ranked before it
  for (int64_t jz = 0; jz < c; ++jz) {
    if (sig[jz] != 0.0) continue;
    double* wz = W + jz * r;
    for (int64_t cand = 0; cand < r; ++cand) {
      for (int64_t q = tid; q < r; q += kSvdThreads) wz[q] = q == cand ? 1.0 : 0.0;
      __syncthreads();
      for (int pass = 0; pass < 2; ++pass) {
        for (int64_t p = 0; p < c; ++p) {
          if (p == jz) continue;
          const bool before = sig[p] > sig[jz] || (sig[p] == sig[jz] && p < jz);
          if (!before) continue;
          const double* wp = W + p * r;
          double d = 0.0;
          for (int64_t q = tid; q < r; q += kSvdThreads) d = fma(wp[q], wz[q], d);
          d = cta_sum(d, red);
          for (int64_t q = tid; q < r; q += kSvdThreads) wz[q] -= d * wp[q];
          __syncthreads();
        }
      }
      double nn = 0.0;
      for (int64_t q = tid; q < r; q += kSvdThreads) nn = fma(wz[q], wz[q], nn);
      nn = cta_sum(nn, red);
      if (nn > 0.25) {
        const double inv = 1.0 / sqrt(nn);
        for (int64_t q = tid; q < r; q += kSvdThreads) wz[q] *= inv;
        __syncthreads();
        break;
      }
      __syncthreads();
    }
  }
  __syncthreads();

  // outputs in descending order
  for (int64_t j = tid; j < c; j += kSvdThreads) {
    int64_t p = 0;
    for (int64_t q = 0; q < c; ++q) p += (sig[q] > sig[j] || (sig[q] == sig[j] && q < j)) ? 1 : 0;
    s[s_off + p] = sig[j];
    pos[j] = static_cast<double>(p);
  }
  __syncthreads();
  // U (m x c) and Vt (c x n), row-major.  Column j of W goes to sorted position p(j).
  for (int64_t e = tid; e < r * c; e += kSvdThreads) {
    const int64_t j = e / r, q = e % r;
    const int64_t p = static_cast<int64_t>(pos[j]);
    if (!trans)
      u[u_off + q * c + p] = W[e];  // W = A: left vectors are U's columns
    else
      vt[vt_off + p * n + q] = W[e];  // W = A^T: left vectors are Vh's rows
  }
  for (int64_t e = tid; e < c * c; e += kSvdThreads) {
    const int64_t j = e / c, q = e % c;
    const int64_t p = static_cast<int64_t>(pos[j]);
    if (!trans)
      vt[vt_off + p * n + q] = V[e];  // right vectors of A are Vh's rows
    else
      u[u_off + q * c + p] = V[e];  // right vectors of A^T are U's columns
  }
  if (tid == 0) info[b] = converged ? 0 : sweep;
}

// One CTA.  sectors: rows of [count, s_off, label, 0] sorted by label; qdim per sector.
// mode: 0 abs, 1 rel, 2 sum2, 3 rsum2, 4 sum1, 5 rsum1; cutoff < 0: no cutoff;
// max_bond < 0: no budget; budget: 0 dense (cost qdim), 1 reduced (cost 1).
// Outputs: keep[sector], sorted_s / sorted_c (global order), stats =
// {kept, dense, discarded, total, kept_w, admissible, T, 0}.
__global__ void __launch_bounds__(kDecideThreads)
decide_kernel(const int64_t* __restrict__ sectors, const double* __restrict__ qdim,
              int64_t n_sec, const double* __restrict__ s, int64_t n_s, double cutoff, int mode,
              double max_bond, int budget, int64_t* __restrict__ keep,
              double* __restrict__ sorted_s, int32_t* __restrict__ sorted_c,
              double* __restrict__ stats) {
  __shared__ int64_t s_begin[257];
  const int tid = threadIdx.x;
  if (n_sec > 256) {
    if (tid == 0) raise_bounds();
    return;
  }
  if (tid == 0) {
    int64_t acc = 0;
    bool ok = true;
    for (int64_t k = 0; k < n_sec; ++k) {
      s_begin[k] = acc;
      const int64_t cnt = sectors[k * kSectorRow], off = sectors[k * kSectorRow + 1];
      ok = ok && cnt >= 0 && off >= 0 && off + cnt <= n_s;
      acc += cnt;
    }
    s_begin[n_sec] = ok ? acc : -1;
    if (!ok) raise_bounds();
  }
  __syncthreads();
  const int64_t T = s_begin[n_sec];
  if (T < 0) return;
  // global rank of every (sigma, sector, index)
  for (int64_t e = tid; e < T; e += kDecideThreads) sorted_c[e] = -1;
  __syncthreads();
  for (int64_t e = tid; e < T; e += kDecideThreads) {
    int64_t k = 0;
    while (k + 1 < n_sec && s_begin[k + 1] <= e) ++k;
    const int64_t i = e - s_begin[k];
    const double v = s[sectors[k * kSectorRow + 1] + i];
    int64_t rank = i;
    for (int64_t o = 0; o < n_sec; ++o) {
      if (o == k) continue;
      const double* so = s + sectors[o * kSectorRow + 1];
      const int64_t cnt = sectors[o * kSectorRow];
      // elements of o before v: those > v, and those == v when o precedes k
      int64_t lo = 0, hi = cnt;
      if (o < k) {
        while (lo < hi) {  // first index with so[idx] < v
          const int64_t mid = (lo + hi) >> 1;
          if (so[mid] >= v) lo = mid + 1; else hi = mid;
        }
      } else {
        while (lo < hi) {  // first index with so[idx] <= v
          const int64_t mid = (lo + hi) >> 1;
          if (so[mid] > v) lo = mid + 1; else hi = mid;
        }
      }
      rank += lo;
    }
    sorted_s[rank] = v;
    sorted_c[rank] = static_cast<int32_t>(k);
  }
  __syncthreads();
  if (tid != 0) return;
  for (int64_t k = 0; k < n_sec; ++k) keep[k] = 0;
  for (int64_t e = 0; e < T; ++e) {
    if (sorted_c[e] < 0 || sorted_c[e] >= n_sec) {  // a NaN breaks the order
      raise_bounds();
      for (int q = 0; q < 8; ++q) stats[q] = 0.0;
      return;
    }
  }
  int64_t adm = T;
  if (cutoff >= 0.0) {
    if (mode == 0 || mode == 1) {
      const double th = mode == 0 ? cutoff : cutoff * (T ? sorted_s[0] : 0.0);
      adm = 0;
      for (int64_t e = 0; e < T; ++e) adm += sorted_s[e] > th ? 1 : 0;
    } else {
      const bool sq = mode == 2 || mode == 3;
      double total = 0.0;
      for (int64_t e = 0; e < T; ++e) {
        const double x = sorted_s[e];
        total += qdim[sorted_c[e]] * (sq ? x * x : x);
      }
      const double th = (mode == 3 || mode == 5) ? cutoff * total : cutoff;
      double dropped = 0.0;
      for (int64_t e = T - 1; e >= 0; --e) {
        const double x = sorted_s[e];
        const double w = qdim[sorted_c[e]] * (sq ? x * x : x);
        if (dropped + w >= th) break;
        dropped += w;
        --adm;
      }
    }
  }
  double used = 0.0, dense = 0.0, kept_w = 0.0;
  int64_t n_kept = 0;
  for (int64_t e = 0; e < adm; ++e) {
    const int32_t k = sorted_c[e];
    const double cost = budget == 0 ? qdim[k] : 1.0;
    if (max_bond >= 0.0 && used + cost > max_bond) break;
    used += cost;
    dense += qdim[k];
    keep[k] += 1;
    kept_w += qdim[k] * sorted_s[e] * sorted_s[e];
    ++n_kept;
  }
  double total2 = 0.0, disc = 0.0;
  for (int64_t e = 0; e < T; ++e) {
    const double x = sorted_s[e];
    total2 += qdim[sorted_c[e]] * x * x;
  }
  for (int64_t e = n_kept; e < T; ++e) {
    const double x = sorted_s[e];
    disc += qdim[sorted_c[e]] * x * x;
  }
  stats[0] = static_cast<double>(n_kept);
  stats[1] = dense;
  stats[2] = disc;
  stats[3] = total2;
  stats[4] = kept_w;
  stats[5] = static_cast<double>(adm);
  stats[6] = static_cast<double>(T);
  stats[7] = 0.0;
}

// rows: [m, n, c (full width), k (kept), u_off, s_off, vt_off, pu_off, ps_off, pv_off, 0, 0]
// U (m x c) -> PU (m x k); S -> PS (k x k diagonal, times scale); Vt (c x n) -> PV (k x n).
// Grid: one CTA per (row, part), part 0..2.
__global__ void __launch_bounds__(256)
svd_compact_kernel(const int64_t* __restrict__ rows, int64_t n_rows, const double* __restrict__ u,
                   int64_t n_u, const double* __restrict__ s, int64_t n_s,
                   const double* __restrict__ vt, int64_t n_vt, double scale,
                   double* __restrict__ pu, int64_t n_pu, double* __restrict__ ps, int64_t n_ps,
                   double* __restrict__ pv, int64_t n_pv) {
  const int64_t b = blockIdx.x / 3, part = blockIdx.x % 3;
  if (b >= n_rows) return;
  const int64_t* row = rows + b * kCompactRow;
  const int64_t m = row[0], n = row[1], c = row[2], k = row[3];
  const int64_t u_off = row[4], s_off = row[5], vt_off = row[6];
  const int64_t pu_off = row[7], ps_off = row[8], pv_off = row[9];
  const bool ok = m >= 0 && n >= 0 && k >= 0 && k <= c && u_off >= 0 && u_off + m * c <= n_u &&
                  s_off >= 0 && s_off + c <= n_s && vt_off >= 0 && vt_off + c * n <= n_vt &&
                  pu_off >= 0 && pu_off + m * k <= n_pu && ps_off >= 0 && ps_off + k * k <= n_ps &&
                  pv_off >= 0 && pv_off + k * n <= n_pv;
  if (!ok) {
    if (threadIdx.x == 0) raise_bounds();
    return;
  }
  if (part == 0) {
    for (int64_t e = threadIdx.x; e < m * k; e += blockDim.x)
      pu[pu_off + e] = u[u_off + (e / k) * c + e % k];
  } else if (part == 1) {
    for (int64_t e = threadIdx.x; e < k * k; e += blockDim.x)
      ps[ps_off + e] = (e / k == e % k) ? s[s_off + e / k] * scale : 0.0;
  } else {
    for (int64_t e = threadIdx.x; e < k * n; e += blockDim.x) pv[pv_off + e] = vt[vt_off + e];
  }
}

static PerDeviceOnce g_svd_opt;
static constexpr int64_t kSvdSmemMaxBytes = 227 * 1024;

}  // namespace tnb

extern "C" int64_t tnb_block_svd_smem_doubles(void) {
  return (tnb::kSvdSmemMaxBytes - 1024) / 8;
}

extern "C" int tnb_block_svd(const int64_t* rows, int64_t n_rows, const double* a, int64_t n_a,
                             double* u, int64_t n_u, double* s, int64_t n_s, double* vt,
                             int64_t n_vt, double* work, int64_t n_work, int32_t* info,
                             int64_t smem_doubles, void* stream) {
  TNB_REQUIRE(n_rows >= 0 && n_a >= 0 && n_u >= 0 && n_s >= 0 && n_vt >= 0 && n_work >= 0,
              "tnb_block_svd: negative size");
  TNB_REQUIRE(smem_doubles >= 0 && smem_doubles <= tnb_block_svd_smem_doubles(),
              "tnb_block_svd: shared-memory request beyond the limit");
  if (n_rows == 0) return TNB_OK;
  TNB_REQUIRE(rows && a && u && s && vt && info && (n_work == 0 || work),
              "tnb_block_svd: null pointer");
  TNB_REQUIRE(n_rows < (1ll << 31), "tnb_block_svd: too many sectors");
  const size_t smem = static_cast<size_t>(smem_doubles) * 8;
  cudaError_t e = tnb::g_svd_opt.once([] {
    return cudaFuncSetAttribute(tnb::block_svd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(tnb::kSvdSmemMaxBytes - 1024));
  });
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_block_svd: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  tnb::block_svd_kernel<<<static_cast<unsigned>(n_rows), tnb::kSvdThreads, smem,
                          tnb::as_stream(stream)>>>(rows, n_rows, a, n_a, u, n_u, s, n_s, vt,
                                                    n_vt, work, n_work, info, smem_doubles);
  return tnb::check_launch("tnb_block_svd");
}

extern "C" int tnb_truncate_decide(const int64_t* sectors, const double* qdim, int64_t n_sec,
                                   const double* s, int64_t n_s, double cutoff, int32_t mode,
                                   double max_bond, int32_t budget, int64_t* keep,
                                   double* sorted_s, int32_t* sorted_c, double* stats,
                                   void* stream) {
  TNB_REQUIRE(n_sec >= 1 && n_sec <= 256, "tnb_truncate_decide: 1..256 sectors");
  TNB_REQUIRE(n_s >= 0 && mode >= 0 && mode <= 5 && (budget == 0 || budget == 1),
              "tnb_truncate_decide: bad mode or size");
  TNB_REQUIRE(sectors && qdim && s && keep && sorted_s && sorted_c && stats,
              "tnb_truncate_decide: null pointer");
  tnb::decide_kernel<<<1, tnb::kDecideThreads, 0, tnb::as_stream(stream)>>>(
      sectors, qdim, n_sec, s, n_s, cutoff, mode, max_bond, budget, keep, sorted_s, sorted_c,
      stats);
  return tnb::check_launch("tnb_truncate_decide");
}

extern "C" int tnb_svd_compact(const int64_t* rows, int64_t n_rows, const double* u, int64_t n_u,
                               const double* s, int64_t n_s, const double* vt, int64_t n_vt,
                               double scale, double* pu, int64_t n_pu, double* ps, int64_t n_ps,
                               double* pv, int64_t n_pv, void* stream) {
  TNB_REQUIRE(n_rows >= 0 && n_u >= 0 && n_s >= 0 && n_vt >= 0 && n_pu >= 0 && n_ps >= 0 &&
                  n_pv >= 0, "tnb_svd_compact: negative size");
  if (n_rows == 0) return TNB_OK;
  TNB_REQUIRE(rows && u && s && vt && pu && ps && pv, "tnb_svd_compact: null pointer");
  TNB_REQUIRE(n_rows < (1ll << 29), "tnb_svd_compact: too many sectors");
  tnb::svd_compact_kernel<<<static_cast<unsigned>(3 * n_rows), 256, 0, tnb::as_stream(stream)>>>(
      rows, n_rows, u, n_u, s, n_s, vt, n_vt, scale, pu, n_pu, ps, n_ps, pv, n_pv);
  return tnb::check_launch("tnb_svd_compact");
}

// ---------------------------------------------------------------------------------------
// Blockwise LQ: the reference's `lq` per coupled sector (ops/linalg.py:549-620), which
// takes the QR of the transpose.  One CTA per sector B (mb x nb, row-major): W = B^T is
// factorised by Householder reflections in LAPACK's convention (dlarfg: beta =
// -sign(alpha) |x|, tau = (beta - alpha) / beta, v(0) = 1; a column with nothing below the
// diagonal gets tau = 0), Q is accumulated backwards from the identity (dorgqr), and the
// outputs are L = R^T (mb x k) and Q^T (k x nb), k = min(mb, nb), both row-major, so the
// gauge is the one the reference's LAPACK QR gives.  The reflector's norm is formed as
// dlapy2 forms it, so a sector whose sub-diagonal part is one element (every sector of a
// multiplicity-one start state) gets LAPACK's bits exactly.

namespace tnb {

constexpr int kQrRow = 8;  // mb, nb, b_off, l_off, q_off, w_off, 0, 0

__global__ void __launch_bounds__(kSvdThreads)
block_lq_kernel(const int64_t* __restrict__ rows, int64_t n_rows, const double* __restrict__ b,
                int64_t n_b, double* __restrict__ lout, int64_t n_l, double* __restrict__ qout,
                int64_t n_q, double* __restrict__ work, int64_t n_work, int64_t smem_doubles) {
  extern __shared__ __align__(16) double qr_smem[];
  __shared__ double red[kSvdWarps];
  const int64_t blk = blockIdx.x;
  if (blk >= n_rows) return;
  const int64_t* row = rows + blk * kQrRow;
  const int64_t mb = row[0], nb = row[1], b_off = row[2], l_off = row[3], q_off = row[4],
                w_off = row[5];
  const int64_t m = nb, n = mb;                 // W = B^T: m x n
  const int64_t k = m < n ? m : n;
  const bool ok = mb >= 0 && nb >= 0 && b_off >= 0 && b_off + mb * nb <= n_b && l_off >= 0 &&
                  l_off + mb * k <= n_l && q_off >= 0 && q_off + k * nb <= n_q &&
                  (w_off >= 0 ? w_off + m * n + m * k + 2 * k <= n_work
                              : m * n + m * k + 2 * k <= smem_doubles);
  if (!ok) {
    if (threadIdx.x == 0) raise_bounds();
    return;
  }
  if (k == 0) return;
  double* W = w_off >= 0 ? work + w_off : qr_smem;  // column j at W + j * m
  double* Q = W + m * n;                             // column j at Q + j * m
  double* tau = Q + m * k;
  double* beta = tau + k;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int64_t e = tid; e < m * n; e += kSvdThreads) {
    const int64_t j = e / m, i = e % m;  // W[i][j] = B[j][i]
    W[e] = b[b_off + j * nb + i];
  }
  __syncthreads();
  for (int64_t j = 0; j < k; ++j) {
    double* wj = W + j * m;
    double x2 = 0.0;
    for (int64_t i = j + 1 + tid; i < m; i += kSvdThreads) x2 = fma(wj[i], wj[i], x2);
    x2 = cta_sum(x2, red);
    const double alpha = wj[j];
    double t = 0.0, bt = alpha, scale = 0.0;
    if (x2 > 0.0) {
      // |(alpha, x)| as LAPACK forms it: xnorm = |x|, then dlapy2(alpha, xnorm) =
      // w sqrt(1 + (z / w)^2) with w = max, z = min, each operation rounded on its own
      const double xnorm = sqrt(x2), aa = fabs(alpha);
      const double w = fmax(aa, xnorm), z = fmin(aa, xnorm);
      const double q = z / w;
      const double nrm = z == 0.0 ? w : __dmul_rn(w, sqrt(__dadd_rn(1.0, __dmul_rn(q, q))));
      bt = alpha >= 0.0 ? -nrm : nrm;
      t = (bt - alpha) / bt;
      scale = 1.0 / (alpha - bt);
    }
    __syncthreads();  // every thread has read alpha
    if (x2 > 0.0)
      for (int64_t i = j + 1 + tid; i < m; i += kSvdThreads) wj[i] *= scale;
    if (tid == 0) {
      tau[j] = t;
      beta[j] = bt;
    }
    __syncthreads();
    if (t != 0.0) {
      // H = I - tau v v^T (v = [1, wj[j+1..]]) on the trailing columns, a warp per column
      for (int64_t c = j + 1 + warp; c < n; c += kSvdWarps) {
        double* wc = W + c * m;
        double d = lane == 0 ? wc[j] : 0.0;
        for (int64_t i = j + 1 + lane; i < m; i += 32) d = fma(wj[i], wc[i], d);
        d = warp_sum(d) * t;
        if (lane == 0) wc[j] -= d;
        for (int64_t i = j + 1 + lane; i < m; i += 32) wc[i] = fma(-d, wj[i], wc[i]);
      }
    }
    __syncthreads();
  }
  // Q = H_0 ... H_{k-1} [I_k; 0], applied from the last reflection back (dorgqr)
  for (int64_t e = tid; e < m * k; e += kSvdThreads) Q[e] = (e / m == e % m) ? 1.0 : 0.0;
  __syncthreads();
  for (int64_t j = k - 1; j >= 0; --j) {
    const double t = tau[j];
    if (t != 0.0) {
      const double* wj = W + j * m;
      for (int64_t c = j + warp; c < k; c += kSvdWarps) {
        double* qc = Q + c * m;
        double d = lane == 0 ? qc[j] : 0.0;
        for (int64_t i = j + 1 + lane; i < m; i += 32) d = fma(wj[i], qc[i], d);
        d = warp_sum(d) * t;
        if (lane == 0) qc[j] -= d;
        for (int64_t i = j + 1 + lane; i < m; i += 32) qc[i] = fma(-d, wj[i], qc[i]);
      }
    }
    __syncthreads();
  }
  // L = R^T (mb x k): L[i][p] = R[p][i] = W[p][i] for p < i, beta on the diagonal
  for (int64_t e = tid; e < mb * k; e += kSvdThreads) {
    const int64_t i = e / k, p = e % k;
    lout[l_off + e] = p < i ? W[i * m + p] : (p == i ? beta[p] : 0.0);
  }
  // Q^T (k x nb): Qt[p][c] = Q[c][p]
  for (int64_t e = tid; e < k * nb; e += kSvdThreads) {
    const int64_t p = e / nb, c = e % nb;
    qout[q_off + e] = Q[p * m + c];
  }
}

static PerDeviceOnce g_lq_opt;

}  // namespace tnb

extern "C" int tnb_block_lq(const int64_t* rows, int64_t n_rows, const double* b, int64_t n_b,
                            double* l, int64_t n_l, double* q, int64_t n_q, double* work,
                            int64_t n_work, int64_t smem_doubles, void* stream) {
  TNB_REQUIRE(n_rows >= 0 && n_b >= 0 && n_l >= 0 && n_q >= 0 && n_work >= 0,
              "tnb_block_lq: negative size");
  TNB_REQUIRE(smem_doubles >= 0 && smem_doubles <= tnb_block_svd_smem_doubles(),
              "tnb_block_lq: shared-memory request beyond the limit");
  if (n_rows == 0) return TNB_OK;
  TNB_REQUIRE(rows && b && l && q && (n_work == 0 || work), "tnb_block_lq: null pointer");
  TNB_REQUIRE(n_rows < (1ll << 31), "tnb_block_lq: too many sectors");
  cudaError_t e = tnb::g_lq_opt.once([] {
    return cudaFuncSetAttribute(tnb::block_lq_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(tnb::kSvdSmemMaxBytes - 1024));
  });
  if (e != cudaSuccess) {
    tnb::set_error(std::string("tnb_block_lq: ") + cudaGetErrorString(e));
    return TNB_ECUDA;
  }
  tnb::block_lq_kernel<<<static_cast<unsigned>(n_rows), tnb::kSvdThreads,
                         static_cast<size_t>(smem_doubles) * 8, tnb::as_stream(stream)>>>(
      rows, n_rows, b, n_b, l, n_l, q, n_q, work, n_work, smem_doubles);
  return tnb::check_launch("tnb_block_lq");
}
