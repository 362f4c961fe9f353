// Host-side preparation of one LP (see pdhg_host.cuh).
#include "pdhg_host.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <queue>
#include <string>
#include <thread>
#include <cstdio>
#include <cstdlib>
#include <sys/stat.h>

namespace sih26 {

bool host_finite_bound(double v) { return !(std::isinf(v) || std::fabs(v) >= 1e30); }

// Runs fn(part, parts) on `parts` host threads (the calling thread takes part 0). The host
// preparation below splits work so that every output element is written by one thread and
// every floating-point sum keeps the reference's order: results do not depend on `parts`.
static int host_parts(long long work) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const long long by_work = std::max(1ll, work / 200000);
  return static_cast<int>(std::min<long long>(std::min(hw, 32u), by_work));
}
template <class F>
static void parallel_parts(int parts, F fn) {
  std::vector<std::thread> pool;
  for (int t = 1; t < parts; ++t) pool.emplace_back(fn, t, parts);
  fn(0, parts);
  for (auto& th : pool) th.join();
}
static inline int split(int count, int part, int parts) {
  return static_cast<int>(static_cast<long long>(count) * part / parts);
}

// farkas_proves_infeasible (src/core/certificate.cpp:29-119) on the ABI's problem: every
// multiplier leans on a bound its row has; d = A'y; the column box reaches at most
// `reachable`; the rows require `required`; a margin beyond 1e-7 (kPrimalFeasibility) of the
// comparison scale proves the LP infeasible. Coefficients of d at 1e-11 (kZeroDrop) of the
// term scale count as zero.
bool farkas_holds(const sankhya_pdhg_problem& p, const std::vector<double>& y) {
  const int m = p.num_rows, n = p.num_cols;
  bool any = false;
  double required = 0.0;
  for (int i = 0; i < m; ++i) {
    if (y[i] != 0.0) any = true;
    if (y[i] > 0.0) {
      if (!host_finite_bound(p.row_lower[i])) return false;
      required += y[i] * p.row_lower[i];
    } else if (y[i] < 0.0) {
      if (!host_finite_bound(p.row_upper[i])) return false;
      required += y[i] * p.row_upper[i];
    }
  }
  if (!any) return false;
  std::vector<double> d(n, 0.0);
  double scale = 0.0;
  for (int j = 0; j < n; ++j) {
    double sum = 0.0;
    for (int k = p.col_starts[j]; k < p.col_starts[j + 1]; ++k) {
      const double term = p.values[k] * y[p.row_indices[k]];
      sum += term;
      scale = std::max(scale, std::fabs(term));
    }
    d[j] = sum;
  }
  double reachable = 0.0;
  for (int j = 0; j < n; ++j) {
    if (d[j] > 1e-11 * std::max(1.0, scale)) {
      if (!host_finite_bound(p.col_upper[j])) return false;
      reachable += d[j] * p.col_upper[j];
    } else if (d[j] < -1e-11 * std::max(1.0, scale)) {
      if (!host_finite_bound(p.col_lower[j])) return false;
      reachable += d[j] * p.col_lower[j];
    }
  }
  const double margin = required - reachable;
  const double comparison = std::max({1.0, std::fabs(required), std::fabs(reachable), scale});
  return margin > 1e-7 * comparison;
}

// ray_proves_unbounded (src/core/certificate.cpp:121-218) for an LP: the direction moves no
// column against a bound it has (beyond 1e-7 of its largest entry), moves no row activity
// against a bound it has (beyond 1e-7 of the term scale), and improves the min-space cost by
// more than 1e-7 of the cost-term scale per unit step.
bool ray_holds(const sankhya_pdhg_problem& p, const std::vector<double>& d) {
  const int m = p.num_rows, n = p.num_cols;
  double magnitude = 0.0;
  for (int j = 0; j < n; ++j) magnitude = std::max(magnitude, std::fabs(d[j]));
  if (magnitude == 0.0) return false;
  const double moving = 1e-7 * magnitude;
  for (int j = 0; j < n; ++j) {
    if (d[j] > moving && host_finite_bound(p.col_upper[j])) return false;
    if (d[j] < -moving && host_finite_bound(p.col_lower[j])) return false;
  }
  std::vector<double> activity(m, 0.0);
  double scale = 0.0;
  for (int j = 0; j < n; ++j) {
    if (d[j] == 0.0) continue;
    for (int k = p.col_starts[j]; k < p.col_starts[j + 1]; ++k) {
      const double term = p.values[k] * d[j];
      activity[p.row_indices[k]] += term;
      scale = std::max(scale, std::fabs(term));
    }
  }
  const double row_moving = 1e-7 * std::max(1.0, scale);
  for (int i = 0; i < m; ++i) {
    if (activity[i] > row_moving && host_finite_bound(p.row_upper[i])) return false;
    if (activity[i] < -row_moving && host_finite_bound(p.row_lower[i])) return false;
  }
  const double sense = p.maximize ? -1.0 : 1.0;
  double improvement = 0.0, cost_scale = 0.0;
  for (int j = 0; j < n; ++j) {
    const double term = sense * p.cost[j] * d[j];
    improvement += term;
    cost_scale = std::max(cost_scale, std::fabs(term));
  }
  return improvement < -1e-7 * std::max(1.0, cost_scale);
}

// Repairs a primal-ray candidate before the exact check. Restarted PDHG on an unbounded LP
// drives the primal weight to its floor, so the dual settles slowly and the last step still
// carries a small movement of the bounded part (a few 1e-6 of the ray) -- above the checker's
// 1e-7. The repair keeps the columns that move by more than 1e-4 of the largest move, drops
// the rest, and projects the kept part onto the null space of the rows it would push against
// a finite bound (modified Gram-Schmidt over those rows), so those activities stay put. Any
// vector that passes ray_holds proves unboundedness, so the repair cannot produce a false
// proof; it returns false when the support is larger than kMaxSupport columns.
bool repair_ray(const sankhya_pdhg_problem& p, std::vector<double>& d) {
  constexpr int kMaxSupport = 256;
  const int n = p.num_cols;
  double mag = 0.0;
  for (int j = 0; j < n; ++j) mag = std::max(mag, std::fabs(d[j]));
  if (mag == 0.0) return false;
  std::vector<int> S;
  for (int j = 0; j < n; ++j) {
    if (std::fabs(d[j]) > 1e-4 * mag) S.push_back(j);
    if (static_cast<int>(S.size()) > kMaxSupport) return false;
  }
  const int k = static_cast<int>(S.size());
  // the rows the support touches, their activity along d, and, as dense rows over the
  // support, those whose activity must stay put: a finite bound on the side the activity moves
  // towards (or either side, for a move at rounding size)
  std::vector<int> row_slot(p.num_rows, -1);
  std::vector<int> touched;
  std::vector<double> act;
  for (int s = 0; s < k; ++s) {
    const int j = S[s];
    for (int t = p.col_starts[j]; t < p.col_starts[j + 1]; ++t) {
      const int i = p.row_indices[t];
      if (row_slot[i] < 0) {
        row_slot[i] = static_cast<int>(touched.size());
        touched.push_back(i);
        act.push_back(0.0);
      }
      act[row_slot[i]] += p.values[t] * d[j];
    }
  }
  double act_max = 0.0;
  for (double v : act) act_max = std::max(act_max, std::fabs(v));
  const double thr = 1e-6 * act_max;
  std::vector<int> keep_slot(touched.size(), -1);
  std::vector<std::vector<double>> rows;
  for (size_t r = 0; r < touched.size(); ++r) {
    const int i = touched[r];
    const bool up_blocked = host_finite_bound(p.row_upper[i]) && act[r] >= -thr;
    const bool down_blocked = host_finite_bound(p.row_lower[i]) && act[r] <= thr;
    if (up_blocked || down_blocked) {
      keep_slot[r] = static_cast<int>(rows.size());
      rows.emplace_back(k, 0.0);
    }
  }
  for (int s = 0; s < k; ++s) {
    const int j = S[s];
    for (int t = p.col_starts[j]; t < p.col_starts[j + 1]; ++t) {
      const int slot = keep_slot[row_slot[p.row_indices[t]]];
      if (slot >= 0) rows[slot][s] = p.values[t];
    }
  }
  // orthonormal basis of the rows' span (modified Gram-Schmidt, rank-revealing threshold)
  std::vector<std::vector<double>> basis;
  for (auto& r : rows) {
    double n0 = 0.0;
    for (double v : r) n0 += v * v;
    n0 = std::sqrt(n0);
    if (n0 == 0.0) continue;
    for (const auto& q : basis) {
      double dot = 0.0;
      for (int s = 0; s < k; ++s) dot += q[s] * r[s];
      for (int s = 0; s < k; ++s) r[s] -= dot * q[s];
    }
    double n1 = 0.0;
    for (double v : r) n1 += v * v;
    n1 = std::sqrt(n1);
    if (n1 <= 1e-10 * n0) continue;
    for (double& v : r) v /= n1;
    basis.push_back(std::move(r));
    if (static_cast<int>(basis.size()) == k) return false;  // no null space left
  }
  std::vector<double> ds(k);
  for (int s = 0; s < k; ++s) ds[s] = d[S[s]];
  for (int pass = 0; pass < 2; ++pass) {  // twice, for the rounding of the first pass
    for (const auto& q : basis) {
      double dot = 0.0;
      for (int s = 0; s < k; ++s) dot += q[s] * ds[s];
      for (int s = 0; s < k; ++s) ds[s] -= dot * q[s];
    }
  }
  std::fill(d.begin(), d.end(), 0.0);
  for (int s = 0; s < k; ++s) d[S[s]] = ds[s];
  return true;
}

static std::string fmtd(const char* f, long long a, long long b = 0) {
  char buf[256];
  std::snprintf(buf, sizeof buf, f, a, b);
  return buf;
}

void check_structure(const sankhya_pdhg_problem& p) {
  const auto bad = [](const std::string& why) {
    throw Failure{SANKHYA_GPU_INVALID_ARGUMENT, why};
  };
  if (p.num_rows < 0 || p.num_cols < 0 || p.num_nonzeros < 0) bad("negative problem size");
  const int m = p.num_rows, n = p.num_cols;
  if (!p.col_starts) bad("col_starts is NULL");
  if (n > 0 && (!p.cost || !p.col_lower || !p.col_upper)) bad("a column array is NULL");
  if (m > 0 && (!p.row_lower || !p.row_upper)) bad("a row array is NULL");
  if (p.num_nonzeros > 0 && (!p.row_indices || !p.values)) bad("matrix arrays are NULL");
  if (p.col_starts[0] != 0) bad("col_starts[0] != 0");
  if (p.col_starts[n] != p.num_nonzeros)
    bad(fmtd("col_starts[n] = %lld but num_nonzeros = %lld", p.col_starts[n], p.num_nonzeros));
  // col_starts first: once it never decreases, every column's range lies in [0, nnz], so the
  // entry checks below read nothing outside the arrays
  for (int j = 0; j < n; ++j)
    if (p.col_starts[j + 1] < p.col_starts[j]) bad(fmtd("col_starts decreases at column %lld", j));
  // the entries, in column ranges on host threads; the first bad column in column order is
  // reported, with the message a single pass would give
  const int parts = host_parts(p.num_nonzeros);
  std::vector<std::string> why(parts);
  parallel_parts(parts, [&](int t, int T) {
    for (int j = split(n, t, T), j1 = split(n, t + 1, T); j < j1; ++j) {
      const int b = p.col_starts[j], e = p.col_starts[j + 1];
      for (int k = b; k < e; ++k) {
        const int i = p.row_indices[k];
        if (i < 0 || i >= m) {
          why[t] = fmtd("row index %lld out of range in column %lld", i, j);
          return;
        }
        if (k > b && i <= p.row_indices[k - 1]) {
          why[t] = fmtd("row indices of column %lld are not strictly ascending (entry %lld)", j, k);
          return;
        }
      }
    }
  });
  for (const std::string& w : why)
    if (!w.empty()) bad(w);
}

std::string validate_model(const sankhya_pdhg_problem& p) {
  char buf[256];
  const int m = p.num_rows, n = p.num_cols;
  // the values, in column ranges on host threads; the first bad entry in column order wins
  const int parts = host_parts(p.num_nonzeros);
  std::vector<long long> first(parts, -1);
  parallel_parts(parts, [&](int t, int T) {
    const long long k0 = p.col_starts[split(n, t, T)], k1 = p.col_starts[split(n, t + 1, T)];
    for (long long k = k0; k < k1; ++k) {
      if (!std::isfinite(p.values[k])) {
        first[t] = k;
        return;
      }
    }
  });
  for (int t = 0; t < parts; ++t) {
    if (first[t] < 0) continue;
    const long long k = first[t];
    const int j = static_cast<int>(std::upper_bound(p.col_starts, p.col_starts + n + 1,
                                                    static_cast<int>(k)) - p.col_starts) - 1;
    std::snprintf(buf, sizeof buf, "matrix entry (%d, %d) is %g, which is not a usable coefficient",
                  p.row_indices[k], j, p.values[k]);
    return buf;
  }
  for (int j = 0; j < n; ++j) {
    const double lo = p.col_lower[j], hi = p.col_upper[j];
    if (std::isnan(lo) || std::isnan(hi)) {
      std::snprintf(buf, sizeof buf, "column %d has a NaN bound", j);
      return buf;
    }
    if (lo > hi) {
      std::snprintf(buf, sizeof buf, "column %d has lower bound %g above upper bound %g", j, lo, hi);
      return buf;
    }
    if (std::isnan(p.cost[j])) {
      std::snprintf(buf, sizeof buf, "column %d has a NaN objective coefficient", j);
      return buf;
    }
  }
  for (int i = 0; i < m; ++i) {
    const double lo = p.row_lower[i], hi = p.row_upper[i];
    if (std::isnan(lo) || std::isnan(hi)) {
      std::snprintf(buf, sizeof buf, "row %d has a NaN bound", i);
      return buf;
    }
    if (lo > hi) {
      std::snprintf(buf, sizeof buf, "row %d has lower bound %g above upper bound %g", i, lo, hi);
      return buf;
    }
  }
  if (std::isnan(p.objective_offset)) return "objective offset is NaN";
  return "";
}

// apply_pass (src/la/scaling.cpp:14-40): the reference rebuilds the matrix through
// add_entry + finalize(0.0), which keeps pattern and order, i.e. value * row_pass * col_pass.
// A row-major copy of the matrix values (each row's entries in ascending column order), kept
// in step with the column-major values: every pass multiplies both copies by the same factors
// in the same order, so they hold the same bits.
struct RowView {
  std::vector<int> ptr, col;
  std::vector<double> val;
};
static RowView row_view(const sankhya_pdhg_problem& p, int parts) {
  RowView r;
  const int m = p.num_rows;
  r.ptr.assign(m + 1, 0);
  for (long long k = 0; k < p.num_nonzeros; ++k) ++r.ptr[p.row_indices[k] + 1];
  for (int i = 0; i < m; ++i) r.ptr[i + 1] += r.ptr[i];
  r.col.resize(p.num_nonzeros);
  r.val.resize(p.num_nonzeros);
  // a thread owns a range of rows and places only their entries
  parallel_parts(parts, [&](int part, int np) {
    const int r0 = split(m, part, np), r1 = split(m, part + 1, np);
    std::vector<int> next(r.ptr.begin() + r0, r.ptr.begin() + r1);
    for (int j = 0; j < p.num_cols; ++j) {
      for (int k = p.col_starts[j]; k < p.col_starts[j + 1]; ++k) {
        const int i = p.row_indices[k];
        if (i < r0 || i >= r1) continue;
        const int t = next[i - r0]++;
        r.col[t] = j;
        r.val[t] = p.values[k];
      }
    }
  });
  return r;
}

static void apply_pass(const sankhya_pdhg_problem& p, Scaling& s, RowView& rv,
                       const std::vector<double>& rp, const std::vector<double>& cp, int parts) {
  parallel_parts(parts, [&](int part, int np) {
    for (int j = split(p.num_cols, part, np); j < split(p.num_cols, part + 1, np); ++j) {
      const double cj = cp[j];
      for (int k = p.col_starts[j]; k < p.col_starts[j + 1]; ++k) {
        s.values[k] = s.values[k] * rp[p.row_indices[k]] * cj;
      }
    }
    for (int i = split(p.num_rows, part, np); i < split(p.num_rows, part + 1, np); ++i) {
      const double ri = rp[i];
      for (int t = rv.ptr[i]; t < rv.ptr[i + 1]; ++t) rv.val[t] = rv.val[t] * ri * cp[rv.col[t]];
    }
  });
  for (int i = 0; i < p.num_rows; ++i) s.dr[i] *= rp[i];
  for (int j = 0; j < p.num_cols; ++j) s.dc[j] *= cp[j];
}

// Per-row and per-column max |a| (Ruiz) or sum |a| (Pock-Chambolle) of the current values.
// Each row and each column is reduced by one thread in ascending order of the other index,
// which is the order the reference accumulates in (column by column, scaling.cpp:44-100), so
// the sums are bit-identical to it whatever the thread count.
static void row_col_norms(const sankhya_pdhg_problem& p, const RowView& rv, const Scaling& s,
                          bool sum, std::vector<double>& ra, std::vector<double>& ca, int parts) {
  const int m = p.num_rows, n = p.num_cols;
  parallel_parts(parts, [&](int part, int np) {
    for (int j = split(n, part, np); j < split(n, part + 1, np); ++j) {
      double acc = 0.0;
      for (int k = p.col_starts[j]; k < p.col_starts[j + 1]; ++k) {
        const double mag = std::fabs(s.values[k]);
        acc = sum ? acc + mag : std::max(acc, mag);
      }
      ca[j] = acc;
    }
    for (int i = split(m, part, np); i < split(m, part + 1, np); ++i) {
      double acc = 0.0;
      for (int t = rv.ptr[i]; t < rv.ptr[i + 1]; ++t) {
        const double mag = std::fabs(rv.val[t]);
        acc = sum ? acc + mag : std::max(acc, mag);
      }
      ra[i] = acc;
    }
  });
}

Scaling build_scaling(const sankhya_pdhg_problem& p, const std::vector<double>& min_cost,
                      int ruiz_rounds) {
  const int m = p.num_rows, n = p.num_cols;
  const int parts = host_parts(p.num_nonzeros);
  Scaling s;
  s.dr.assign(m, 1.0);
  s.dc.assign(n, 1.0);
  s.values.assign(p.values, p.values + p.num_nonzeros);
  std::vector<double> ra(m), ca(n), rp(m), cp(n);
  RowView rv = row_view(p, parts);
  // ruiz_round (scaling.cpp:44-72): 1/sqrt(max |a|) per row and column
  for (int round = 0; round < ruiz_rounds; ++round) {
    row_col_norms(p, rv, s, false, ra, ca, parts);
    for (int i = 0; i < m; ++i) rp[i] = ra[i] > 0.0 ? 1.0 / std::sqrt(ra[i]) : 1.0;
    for (int j = 0; j < n; ++j) cp[j] = ca[j] > 0.0 ? 1.0 / std::sqrt(ca[j]) : 1.0;
    apply_pass(p, s, rv, rp, cp, parts);
  }
  // pock_chambolle_round (scaling.cpp:76-100), alpha = 1: 1/sqrt(sum |a|)
  row_col_norms(p, rv, s, true, ra, ca, parts);
  for (int i = 0; i < m; ++i) rp[i] = ra[i] > 0.0 ? 1.0 / std::sqrt(ra[i]) : 1.0;
  for (int j = 0; j < n; ++j) cp[j] = ca[j] > 0.0 ? 1.0 / std::sqrt(ca[j]) : 1.0;
  apply_pass(p, s, rv, rp, cp, parts);
  // vectors (scaling.cpp:124-145); scale_bound multiplies by 1/dc, it does not divide
  s.cost.resize(n);
  s.cl.resize(n);
  s.cu.resize(n);
  for (int j = 0; j < n; ++j) {
    const double dc = s.dc[j];
    s.cost[j] = min_cost[j] * dc;
    s.cl[j] = host_finite_bound(p.col_lower[j]) ? p.col_lower[j] * (1.0 / dc) : p.col_lower[j];
    s.cu[j] = host_finite_bound(p.col_upper[j]) ? p.col_upper[j] * (1.0 / dc) : p.col_upper[j];
  }
  s.rl.resize(m);
  s.ru.resize(m);
  for (int i = 0; i < m; ++i) {
    const double dr = s.dr[i];
    s.rl[i] = host_finite_bound(p.row_lower[i]) ? p.row_lower[i] * dr : p.row_lower[i];
    s.ru[i] = host_finite_bound(p.row_upper[i]) ? p.row_upper[i] * dr : p.row_upper[i];
  }
  return s;
}

// Positions sorted by count, largest first, ties in index order (a stable counting sort).
static std::vector<int> order_by_count_desc(const std::vector<int>& count) {
  int top = 0;
  for (int c : count) top = std::max(top, c);
  std::vector<int> start(static_cast<size_t>(top) + 2, 0);
  for (int c : count) ++start[top - c + 1];
  for (int b = 1; b <= top + 1; ++b) start[b] += start[b - 1];
  std::vector<int> order(count.size());
  for (int i = 0; i < static_cast<int>(count.size()); ++i) order[start[top - count[i]]++] = i;
  return order;
}

PermutedLp permute(const sankhya_pdhg_problem& p, const std::vector<double>& v) {
  PermutedLp q;
  const int m = p.num_rows, n = p.num_cols;
  const int parts = host_parts(p.num_nonzeros);
  q.m = m;
  q.n = n;
  q.nnz = p.num_nonzeros;
  std::vector<int> rc(m, 0), cc(n, 0);
  for (int j = 0; j < n; ++j) cc[j] = p.col_starts[j + 1] - p.col_starts[j];
  for (long long k = 0; k < q.nnz; ++k) ++rc[p.row_indices[k]];
  q.row_perm = order_by_count_desc(rc);
  q.col_perm = order_by_count_desc(cc);
  std::vector<int> row_pos(m), col_pos(n);
  for (int t = 0; t < m; ++t) row_pos[q.row_perm[t]] = t;
  for (int t = 0; t < n; ++t) col_pos[q.col_perm[t]] = t;
  // A: rows in permuted order; walking permuted columns in order keeps each row ascending.
  // A thread owns a range of permuted rows and places only their entries.
  q.a_ptr.assign(m + 1, 0);
  for (int t = 0; t < m; ++t) q.a_ptr[t + 1] = q.a_ptr[t] + rc[q.row_perm[t]];
  q.a_idx.resize(q.nnz);
  q.a_val.resize(q.nnz);
  parallel_parts(parts, [&](int part, int np) {
    const int r0 = split(m, part, np), r1 = split(m, part + 1, np);
    std::vector<int> next(q.a_ptr.begin() + r0, q.a_ptr.begin() + r1);
    for (int t = 0; t < n; ++t) {
      const int j = q.col_perm[t];
      for (int k = p.col_starts[j]; k < p.col_starts[j + 1]; ++k) {
        const int r = row_pos[p.row_indices[k]];
        if (r < r0 || r >= r1) continue;
        const int slot = next[r - r0]++;
        q.a_idx[slot] = t;
        q.a_val[slot] = v[k];
      }
    }
  });
  // A': rows are permuted columns; walking permuted rows in order keeps each ascending
  q.at_ptr.assign(n + 1, 0);
  for (int t = 0; t < n; ++t) q.at_ptr[t + 1] = q.at_ptr[t] + cc[q.col_perm[t]];
  q.at_idx.resize(q.nnz);
  q.at_val.resize(q.nnz);
  parallel_parts(parts, [&](int part, int np) {
    const int c0 = split(n, part, np), c1 = split(n, part + 1, np);
    std::vector<int> next(q.at_ptr.begin() + c0, q.at_ptr.begin() + c1);
    for (int t = 0; t < m; ++t) {
      for (int k = q.a_ptr[t]; k < q.a_ptr[t + 1]; ++k) {
        const int c = q.a_idx[k];
        if (c < c0 || c >= c1) continue;
        const int slot = next[c - c0]++;
        q.at_idx[slot] = t;
        q.at_val[slot] = q.a_val[k];
      }
    }
  });
  return q;
}

sankhya_pdhg_quality quality_from_slots(const double* q, double objective, double dual_bound) {
  sankhya_pdhg_quality r{};
  r.primal_infeasibility = q[0];
  r.primal_infeasibility_scaled = q[1];
  r.dual_infeasibility = q[2];
  const double price_scale = std::max(1.0, q[7]);
  r.dual_infeasibility_scaled = std::max(q[3], std::max(q[5], q[6]) / price_scale);
  r.complementarity_violation = q[4];
  r.absolute_gap = std::fabs(objective - dual_bound);
  r.relative_gap = r.absolute_gap / std::max(1.0, std::fabs(objective));
  return r;
}

static int lanes_for(int len, int nnz_per_lane) {
  // smallest power of two with at most nnz_per_lane nonzeros per lane, capped at a warp
  int lanes = 1;
  while (lanes < 32 && lanes * nnz_per_lane < len) lanes *= 2;
  return lanes;
}

// A warp works through its items one after another and each costs about one round of
// dependent memory latency, whatever its length, so the balance counts work units: one per
// item or segment, plus a small term for its nonzeros.
static double unit_cost(int nnz) { return 1.0 + nnz / 2048.0; }

HostPart partition(const std::vector<int>& ptr, int G, int warps_per_block, int lanes_override,
                   Schedule sched, bool sliced) {
  constexpr int kSeg = 512;        // == kSegment in pdhg_kernels.cuh
  constexpr int kItem = 512;       // == kItemNnz
  // rows up to this length go to stream items (at most kStreamRowMax = 32 rows per item)
  const int kStreamRow = std::max(1, std::min(sched.stream_row_max, 32));
  const int npl = std::max(1, sched.nnz_per_lane);
  (void)warps_per_block;
  const int rows = static_cast<int>(ptr.size()) - 1;
  const auto len = [&](int r) { return ptr[r + 1] - ptr[r]; };
  // long rows: the prefix longer than one item (rows are sorted longest first)
  int L = 0;
  while (L < rows && len(L) > kItem) ++L;
  // items of short rows: grouped (one lane group per row) for rows longer than kStreamRow or
  // when a lane count is forced; stream items for the rest
  std::vector<int4> items;
  std::vector<double> item_cost;
  long long sell_entries = 0;
  for (int r = L; r < rows;) {
    if (lanes_override > 0 || len(r) > kStreamRow) {
      const int lanes = lanes_override > 0 ? lanes_override : lanes_for(len(r), npl);
      const int per = 32 / lanes;
      const int begin = r;
      int nnz = 0;
      while (r < rows && r - begin < per &&
             (lanes_override > 0 || (len(r) > kStreamRow && lanes_for(len(r), npl) == lanes))) {
        nnz += len(r);
        ++r;
      }
      items.push_back(make_int4(begin, r, lanes, 0));
      item_cost.push_back(unit_cost(nnz));
    } else if (sliced) {
      // a slice: up to 32 consecutive short rows, padded to the longest of them
      const int begin = r;
      int nnz = 0, longest = 0;
      while (r < rows && r - begin < 32 && len(r) <= kStreamRow) {
        nnz += len(r);
        longest = std::max(longest, len(r));
        ++r;
      }
      longest = std::max(longest, 1);
      items.push_back(make_int4(begin, r, -longest, static_cast<int>(sell_entries)));
      sell_entries += static_cast<long long>(r - begin) * longest;
      item_cost.push_back(unit_cost(nnz));
    } else {
      const int begin = r;
      int nnz = 0;
      while (r < rows && r - begin < 32 && nnz + len(r) <= kItem) {
        nnz += len(r);
        ++r;
      }
      items.push_back(make_int4(begin, r, 0, 0));
      item_cost.push_back(unit_cost(nnz));
    }
  }
  if (sell_entries > 0x7fffffffLL)
    throw Failure{SANKHYA_GPU_INVALID_ARGUMENT, "slice arrays exceed 2^31 entries"};
  // work of each long row: its segments plus the segment-sum step
  double total = 0.0;
  std::vector<double> long_cost(L);
  for (int r = 0; r < L; ++r) {
    const int segs = (len(r) + kSeg - 1) / kSeg;
    long_cost[r] = segs * unit_cost(kSeg) + 0.5;
    total += long_cost[r];
  }
  for (double c : item_cost) total += c;
  const double target = total / G;
  // LPT assignment of long rows to blocks
  std::vector<double> load(G, 0.0);
  std::vector<std::vector<int>> blk_long(G);
  using Entry = std::pair<double, int>;
  std::priority_queue<Entry, std::vector<Entry>, std::greater<Entry>> heap;
  for (int b = 0; b < G; ++b) heap.push({0.0, b});
  for (int r = 0; r < L; ++r) {
    auto [l, b] = heap.top();
    heap.pop();
    blk_long[b].push_back(r);
    load[b] = l + long_cost[r];
    heap.push({load[b], b});
  }
  HostPart hp;
  hp.blk_seg_begin.assign(G + 1, 0);
  hp.blk_long_begin.assign(G + 1, 0);
  for (int b = 0; b < G; ++b) {
    for (int r : blk_long[b]) {
      const int first = static_cast<int>(hp.segs.size());
      int count = 0;
      for (int k = ptr[r]; k < ptr[r + 1]; k += kSeg) {
        hp.segs.push_back(make_int4(r, k, std::min(k + kSeg, ptr[r + 1]), 0));
        ++count;
      }
      hp.longs.push_back(make_int4(r, first, count, 0));
    }
    hp.blk_seg_begin[b + 1] = static_cast<int>(hp.segs.size());
    hp.blk_long_begin[b + 1] = static_cast<int>(hp.longs.size());
  }
  // items go one by one, in row order, to the least-loaded block (long rows included in
  // the loads), so every block gets a similar mix of item kinds; each block's items are then
  // stored contiguously, in row order
  std::vector<int> owner(items.size());
  {
    std::priority_queue<Entry, std::vector<Entry>, std::greater<Entry>> h2;
    for (int b = 0; b < G; ++b) h2.push({load[b], b});
    for (size_t i = 0; i < items.size(); ++i) {
      auto [l, b] = h2.top();
      h2.pop();
      owner[i] = b;
      h2.push({l + item_cost[i], b});
    }
  }
  hp.blk_item_begin.assign(G + 1, 0);
  for (size_t i = 0; i < items.size(); ++i) ++hp.blk_item_begin[owner[i] + 1];
  for (int b = 0; b < G; ++b) hp.blk_item_begin[b + 1] += hp.blk_item_begin[b];
  std::vector<int4> ordered(items.size());
  std::vector<int> fill(hp.blk_item_begin.begin(), hp.blk_item_begin.end() - 1);
  for (size_t i = 0; i < items.size(); ++i) ordered[fill[owner[i]]++] = items[i];
  items.swap(ordered);
  (void)target;
  hp.items = std::move(items);
  hp.sell_entries = sell_entries;
  return hp;
}

// ---- autotuner key and cache --------------------------------------------------------------

static std::string sig2(double v) {  // two significant digits
  char b[32];
  std::snprintf(b, sizeof b, "%.2g", v);
  return b;
}

static std::string length_stats(const std::vector<int>& ptr) {
  const int rows = static_cast<int>(ptr.size()) - 1;
  if (rows <= 0) return "empty";
  double sum = 0.0, sq = 0.0, nnz_long = 0.0, nnz_mid = 0.0;
  int mx = 0;
  for (int r = 0; r < rows; ++r) {
    const int len = ptr[r + 1] - ptr[r];
    sum += len;
    sq += static_cast<double>(len) * len;
    mx = std::max(mx, len);
    if (len > 512) nnz_long += len;
    else if (len > 32) nnz_mid += len;
  }
  const double mean = sum / rows;
  const double cv = mean > 0.0 ? std::sqrt(std::max(0.0, sq / rows - mean * mean)) / mean : 0.0;
  const double tot = std::max(1.0, sum);
  // fractions of the nonzeros in 33-512 and >512 nonzero rows, in steps of 0.05
  const auto step = [](double f) { return sig2(std::round(f * 20.0) / 20.0); };
  return "mean" + sig2(mean) + ",max" + sig2(mx) + ",cv" + sig2(cv) + ",mid" + step(nnz_mid / tot) +
         ",long" + step(nnz_long / tot);
}

std::string autotune_key(const PermutedLp& q, int G, int sms, int value_bytes) {
  const auto log2b = [](long long v) {
    int b = 0;
    while ((1ll << b) < v) ++b;
    return std::to_string(b);
  };
  return "sm" + std::to_string(sms) + "|G" + std::to_string(G) + "|v" + std::to_string(value_bytes) +
         "|m2^" + log2b(q.m) + "|n2^" + log2b(q.n) + "|nnz2^" + log2b(q.nnz) + "|rows:" +
         length_stats(q.a_ptr) + "|cols:" + length_stats(q.at_ptr);
}

std::string autotune_cache_path() {
  if (const char* e = std::getenv("SANKHYA_PDHG_AUTOTUNE_CACHE")) return e;
  if (const char* x = std::getenv("XDG_CACHE_HOME")) return std::string(x) + "/sih26_b200/autotune.tsv";
  if (const char* h = std::getenv("HOME")) return std::string(h) + "/.cache/sih26_b200/autotune.tsv";
  return "sih26_b200_autotune.tsv";
}

// One line per key: key, then stream_row_max and nnz_per_lane for A and for A'. The last line
// of a key wins.
bool autotune_lookup(const std::string& path, const std::string& key, Schedule* a, Schedule* at) {
  std::FILE* f = std::fopen(path.c_str(), "r");
  if (!f) return false;
  bool found = false;
  char line[1024];
  while (std::fgets(line, sizeof line, f)) {
    char* tab = std::strchr(line, '\t');
    if (!tab) continue;
    if (std::string(line, tab - line) != key) continue;
    Schedule x, y;
    if (std::sscanf(tab + 1, "%d\t%d\t%d\t%d", &x.stream_row_max, &x.nnz_per_lane,
                    &y.stream_row_max, &y.nnz_per_lane) == 4 &&
        x.stream_row_max > 0 && x.nnz_per_lane > 0 && y.stream_row_max > 0 && y.nnz_per_lane > 0) {
      *a = x;
      *at = y;
      found = true;
    }
  }
  std::fclose(f);
  return found;
}

void autotune_store(const std::string& path, const std::string& key, const Schedule& a,
                    const Schedule& at, double us_a, double us_at) {
  const size_t slash = path.find_last_of('/');
  if (slash != std::string::npos) {  // create the directory chain (best effort)
    for (size_t k = path.find('/', 1); k != std::string::npos && k <= slash; k = path.find('/', k + 1))
      ::mkdir(path.substr(0, k).c_str(), 0755);
  }
  std::FILE* f = std::fopen(path.c_str(), "a");
  if (!f) return;
  std::fprintf(f, "%s\t%d\t%d\t%d\t%d\t%.2f\t%.2f\n", key.c_str(), a.stream_row_max,
               a.nnz_per_lane, at.stream_row_max, at.nnz_per_lane, us_a, us_at);
  std::fclose(f);
}

bool chunk_lookup(const std::string& path, const std::string& key, long long* chunk) {
  std::FILE* f = std::fopen(path.c_str(), "r");
  if (!f) return false;
  bool found = false;
  char line[1024];
  while (std::fgets(line, sizeof line, f)) {
    char* tab = std::strchr(line, '\t');
    if (!tab) continue;
    if (std::string(line, tab - line) != key) continue;
    long long v = 0;
    if (std::sscanf(tab + 1, "%lld", &v) == 1 && v > 0) {
      *chunk = v;
      found = true;
    }
  }
  std::fclose(f);
  return found;
}

void chunk_store(const std::string& path, const std::string& key, long long chunk, double rate) {
  const size_t slash = path.find_last_of('/');
  if (slash != std::string::npos) {
    for (size_t k = path.find('/', 1); k != std::string::npos && k <= slash; k = path.find('/', k + 1))
      ::mkdir(path.substr(0, k).c_str(), 0755);
  }
  std::FILE* f = std::fopen(path.c_str(), "a");
  if (!f) return;
  std::fprintf(f, "%s\t%lld\t%.4g\n", key.c_str(), chunk, rate);
  std::fclose(f);
}

std::string chunk_key(int sms, int slots, std::vector<long long> nnz, std::vector<double> per_row) {
  const auto median = [](auto v) {
    if (v.empty()) return 0.0;
    std::nth_element(v.begin(), v.begin() + v.size() / 2, v.end());
    return static_cast<double>(v[v.size() / 2]);
  };
  const double mn = median(nnz), mr = median(per_row);
  int b = 0;
  while (std::ldexp(1.0, b) < mn) ++b;
  return "served|sm" + std::to_string(sms) + "|slots" + std::to_string(slots) + "|nnz2^" +
         std::to_string(b) + "|perrow" + sig2(mr);
}

// mt19937 (Matsumoto & Nishimura) and libstdc++'s generate_canonical<double, 53> for a
// 32-bit engine: (g0 + g1 * 2^32) / 2^64, clamped below 1.
void uniform_draws(uint32_t seed, double lo, double hi, size_t count, double* out) {
  uint32_t st[624];
  st[0] = seed;
  for (int k = 1; k < 624; ++k) st[k] = 1812433253u * (st[k - 1] ^ (st[k - 1] >> 30)) + k;
  int index = 624;
  const auto next = [&]() {
    if (index >= 624) {
      for (int k = 0; k < 624; ++k) {
        const uint32_t y = (st[k] & 0x80000000u) | (st[(k + 1) % 624] & 0x7fffffffu);
        st[k] = st[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
      }
      index = 0;
    }
    uint32_t y = st[index++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
  };
  for (size_t t = 0; t < count; ++t) {
    double sum = 0.0, tmp = 1.0;
    for (int k = 0; k < 2; ++k) {
      sum += static_cast<double>(next()) * tmp;
      tmp *= 4294967296.0;
    }
    double r = sum / tmp;
    if (r >= 1.0) r = std::nextafter(1.0, 0.0);
    out[t] = (r * (hi - lo)) + lo;
  }
}

}  // namespace sih26
