// Host-side planner kernels of the tenet_b200 library: plain C++ over host arrays, no
// device.  They replace the per-block Python loops of the table builder:
//   tnb_plan_gather_rows  one descriptor row per destination block (dims ordered by
//                         destination stride, extent-1 dims dropped, contiguous dims merged);
//   tnb_plan_gather_table a block map's whole gather table: terms grouped by destination
//                         block, one row per block with terms, then zero-writing rows;
//   tnb_plan_compose      the sparse product of two block maps (ops/repartition.py:298-316).
#include <stdint.h>

#include <algorithm>
#include <numeric>
#include <unordered_map>
#include <vector>

#include "tenet_b200.h"

namespace {
constexpr int kSegW = TNB_SEG_WIDTH;
constexpr int kMaxRank = TNB_MAX_RANK;
}  // namespace

namespace {

// One descriptor row: dims ordered by destination stride (ties: source column, then row
// stride; stable), extent-1 dims dropped, contiguous dims merged.
int build_row(int nd, const int64_t* D, const int64_t* A, const int64_t* B, const int64_t* C,
              int64_t d_off, int64_t size, int64_t t_begin, int64_t t_end, int64_t buf,
              std::vector<int>& order, int64_t* row) {
  order.resize(nd);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    if (A[x] != A[y]) return A[x] > A[y];
    if (C[x] != C[y]) return C[x] > C[y];
    return B[x] > B[y];
  });
  int64_t od[kMaxRank], oa[kMaxRank], ob[kMaxRank], oc[kMaxRank];
  int n = 0;
  for (int k : order) {
    const int64_t d = D[k], a = A[k], b = B[k], c = C[k];
    if (d == 1) continue;
    if (n > 0 && oa[n - 1] == a * d && ob[n - 1] == b * d && oc[n - 1] == c * d) {
      od[n - 1] *= d;
      oa[n - 1] = a;
      ob[n - 1] = b;
      oc[n - 1] = c;
      continue;
    }
    if (n == kMaxRank) return TNB_EINVAL;  // a block of rank above the kernel's limit
    od[n] = d;
    oa[n] = a;
    ob[n] = b;
    oc[n] = c;
    ++n;
  }
  if (n == 0) {
    od[0] = 1;
    oa[0] = 1;
    ob[0] = 0;
    oc[0] = 0;
    n = 1;
  }
  std::fill(row, row + kSegW, int64_t{0});
  row[0] = d_off;
  row[1] = size;
  row[2] = n;
  row[3] = t_begin;
  row[4] = t_end;
  row[5] = buf;
  for (int k = 0; k < n; ++k) {
    row[8 + k] = od[k];
    row[16 + k] = oa[k];
    row[24 + k] = ob[k];
    row[32 + k] = oc[k];
  }
  return TNB_OK;
}

}  // namespace

extern "C" int tnb_plan_gather_rows(int64_t n_rows, int32_t nd, const int64_t* dims,
                                    const int64_t* dstr, const int64_t* rstr,
                                    const int64_t* cstr, const int64_t* d_off,
                                    const int64_t* sizes, const int64_t* t_begin,
                                    const int64_t* t_end, int64_t buf, int64_t* rows) {
  if (n_rows < 0 || nd < 0 || nd > 64) return TNB_EINVAL;
  if (n_rows > 0 && (!dims || !dstr || !rstr || !cstr || !d_off || !sizes || !t_begin ||
                     !t_end || !rows))
    return TNB_EINVAL;
  std::vector<int> order;
  for (int64_t r = 0; r < n_rows; ++r) {
    const int rc = build_row(nd, dims + r * nd, dstr + r * nd, rstr + r * nd, cstr + r * nd,
                             d_off[r], sizes[r], t_begin[r], t_end[r], buf, order,
                             rows + r * kSegW);
    if (rc != TNB_OK) return rc;
  }
  return TNB_OK;
}

extern "C" int tnb_plan_gather_table(int64_t n_terms, const int64_t* t_src,
                                     const int64_t* t_dst, const double* t_coef, int64_t n_src,
                                     const int64_t* s_off, const int64_t* s_ld,
                                     const int64_t* s_rs, const int64_t* s_cs, int64_t n_dst,
                                     const int64_t* d_off, const int64_t* d_str,
                                     const int64_t* d_shape, const int64_t* d_size,
                                     const uint8_t* keep, int32_t nd, const int64_t* perm,
                                     int64_t buf, int64_t* rows, int64_t* out_src,
                                     double* out_coef, int64_t* out_ld, int64_t* counts) {
  if (n_terms < 0 || n_src < 0 || n_dst < 0 || nd < 0 || nd > 64 || !counts) return TNB_EINVAL;
  if ((n_terms && (!t_src || !t_dst || !t_coef || !out_src || !out_coef || !out_ld)) ||
      (n_src && (!s_off || !s_ld || (nd && (!s_rs || !s_cs)))) ||
      (n_dst && (!d_off || !d_size || !keep || !rows || (nd && (!d_str || !d_shape)))) ||
      (nd && !perm))
    return TNB_EINVAL;
  for (int k = 0; k < nd; ++k)
    if (perm[k] < 0 || perm[k] >= nd) return TNB_EINVAL;
  std::vector<uint8_t> covered(static_cast<size_t>(n_dst), 0);
  std::vector<int64_t> sel;
  sel.reserve(static_cast<size_t>(n_terms));
  for (int64_t t = 0; t < n_terms; ++t) {
    if (t_src[t] < 0 || t_src[t] >= n_src || t_dst[t] < 0 || t_dst[t] >= n_dst)
      return TNB_EINVAL;
    covered[t_dst[t]] = 1;
    if (keep[t_dst[t]]) sel.push_back(t);
  }
  // kept terms grouped by destination block, given order kept inside a group
  std::stable_sort(sel.begin(), sel.end(),
                   [&](int64_t x, int64_t y) { return t_dst[x] < t_dst[y]; });
  const int64_t nt = static_cast<int64_t>(sel.size());
  for (int64_t q = 0; q < nt; ++q) {
    const int64_t t = sel[q];
    out_src[q] = s_off[t_src[t]];
    out_coef[q] = t_coef[t];
    out_ld[q] = s_ld[t_src[t]];
  }
  std::vector<int> order;
  std::vector<int64_t> rs(nd), cs(nd);
  int64_t n_rows = 0;
  for (int64_t q = 0; q < nt;) {  // one row per destination block with terms
    const int64_t j = t_dst[sel[q]], i0 = t_src[sel[q]];
    int64_t e = q;
    while (e < nt && t_dst[sel[e]] == j) ++e;
    for (int k = 0; k < nd; ++k) {  // the first term's source strides, permuted
      rs[k] = s_rs[i0 * nd + perm[k]];
      cs[k] = s_cs[i0 * nd + perm[k]];
    }
    const int rc = build_row(nd, d_shape + j * nd, d_str + j * nd, rs.data(), cs.data(),
                             d_off[j], d_size[j], q, e, buf, order, rows + n_rows * kSegW);
    if (rc != TNB_OK) return rc;
    ++n_rows;
    q = e;
  }
  std::fill(rs.begin(), rs.end(), int64_t{0});
  for (int64_t j = 0; j < n_dst; ++j) {  // then one zero-writing row per uncovered block
    if (covered[j] || !keep[j]) continue;
    const int rc = build_row(nd, d_shape + j * nd, d_str + j * nd, rs.data(), rs.data(),
                             d_off[j], d_size[j], nt, nt, buf, order, rows + n_rows * kSegW);
    if (rc != TNB_OK) return rc;
    ++n_rows;
  }
  counts[0] = n_rows;
  counts[1] = nt;
  return TNB_OK;
}

extern "C" int64_t tnb_plan_compose(int64_t n_a, const double* a, int64_t n_b, const double* b,
                                    double* out, int64_t cap) {
  if (n_a < 0 || n_b < 0 || cap < 0) return -1;
  if ((n_a && !a) || (n_b && !b) || (cap && !out)) return -1;
  // following terms grouped by source, original order kept inside a group
  std::vector<int64_t> order(n_b);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
    return static_cast<int64_t>(b[3 * x]) < static_cast<int64_t>(b[3 * y]);
  });
  std::unordered_map<int64_t, std::pair<int64_t, int64_t>> group;  // src -> [lo, hi)
  group.reserve(static_cast<size_t>(n_b) * 2 + 1);
  for (int64_t i = 0; i < n_b;) {
    const int64_t s = static_cast<int64_t>(b[3 * order[i]]);
    int64_t j = i;
    while (j < n_b && static_cast<int64_t>(b[3 * order[j]]) == s) ++j;
    group[s] = {i, j};
    i = j;
  }
  struct PairHash {
    size_t operator()(const std::pair<int64_t, int64_t>& p) const {
      return std::hash<int64_t>()(p.first * 1000003 + p.second);
    }
  };
  std::unordered_map<std::pair<int64_t, int64_t>, int64_t, PairHash> slot;
  slot.reserve(static_cast<size_t>(n_a) * 2 + 1);
  int64_t n_out = 0;
  for (int64_t t = 0; t < n_a; ++t) {
    const int64_t s = static_cast<int64_t>(a[3 * t]);
    const int64_t m = static_cast<int64_t>(a[3 * t + 1]);
    const double c = a[3 * t + 2];
    auto g = group.find(m);
    if (g == group.end()) continue;
    for (int64_t q = g->second.first; q < g->second.second; ++q) {
      const int64_t f = order[q];
      const int64_t d = static_cast<int64_t>(b[3 * f + 1]);
      const double v = c * b[3 * f + 2];
      auto it = slot.find({s, d});
      if (it == slot.end()) {
        if (n_out >= cap) return -2;  // caller's buffer too small
        slot.emplace(std::make_pair(s, d), n_out);
        out[3 * n_out] = static_cast<double>(s);
        out[3 * n_out + 1] = static_cast<double>(d);
        out[3 * n_out + 2] = 0.0 + v;
        ++n_out;
      } else {
        out[3 * it->second + 2] += v;
      }
    }
  }
  return n_out;
}
