/* TEST INFRASTRUCTURE ONLY -- the oracle (see pdhg_oracle.h). Never linked into the product.
 *
 * Plain C11, FP64, single-threaded. Each routine restates the reference routine it names, in
 * the reference's order of floating-point operations, so that it can be pinned bit for bit
 * against the reference built from its own sources (oracle/Makefile target `ref`). */
#include "pdhg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- helpers: include/sankhya/types.hpp:32-39, the std:: algorithms as libstdc++ has them */

static int is_finite_bound(double v) { return !(isinf(v) || fabs(v) >= 1e30); }
static double dmin(double a, double b) { return (b < a) ? b : a; }          /* std::min */
static double dmax(double a, double b) { return (a < b) ? b : a; }          /* std::max */
static double dclamp(double v, double lo, double hi) {                      /* std::clamp */
  return (v < lo) ? lo : ((hi < v) ? hi : v);
}

/* src/pdhg/pdhg.cpp:63-67 */
static double project(double value, double lower, double upper) {
  if (is_finite_bound(lower) && value < lower) return lower;
  if (is_finite_bound(upper) && value > upper) return upper;
  return value;
}

/* ---- mt19937 (Matsumoto & Nishimura 1998) and generate_canonical<double,53> as libstdc++
 *      implements it for a 32-bit engine: two draws, g0 + g1 * 2^32, divided by 2^64. */

typedef struct { uint32_t s[624]; int i; } mt19937;

static void mt_seed(mt19937* g, uint32_t seed) {
  g->s[0] = seed;
  for (int k = 1; k < 624; ++k) {
    g->s[k] = 1812433253u * (g->s[k - 1] ^ (g->s[k - 1] >> 30)) + (uint32_t)k;
  }
  g->i = 624;
}

static uint32_t mt_next(mt19937* g) {
  if (g->i >= 624) {
    for (int k = 0; k < 624; ++k) {
      const uint32_t y = (g->s[k] & 0x80000000u) | (g->s[(k + 1) % 624] & 0x7fffffffu);
      g->s[k] = g->s[(k + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    g->i = 0;
  }
  uint32_t y = g->s[g->i++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

static double canonical(mt19937* g) {
  double sum = 0.0, tmp = 1.0;
  for (int k = 0; k < 2; ++k) {
    sum += (double)mt_next(g) * tmp;
    tmp *= 4294967296.0;
  }
  double r = sum / tmp;
  if (r >= 1.0) r = nextafter(1.0, 0.0);
  return r;
}

void oracle_uniform_draws(uint32_t seed, double lo, double hi, int64_t count, double* out) {
  mt19937 g;
  mt_seed(&g, seed);
  for (int64_t k = 0; k < count; ++k) out[k] = (canonical(&g) * (hi - lo)) + lo;
}

/* ---- sparse kernels: src/la/sparse.cpp:202-239 ---------------------------------------- */

/* y = A x   (multiply: fill 0 then multiply_add with alpha 1, skipping zero x_j) */
static void csc_multiply(int32_t m, int32_t n, const int32_t* cs, const int32_t* ri,
                         const double* v, const double* x, double* y) {
  for (int32_t i = 0; i < m; ++i) y[i] = 0.0;
  for (int32_t j = 0; j < n; ++j) {
    const double xj = 1.0 * x[j];
    if (xj == 0.0) continue;
    for (int32_t k = cs[j]; k < cs[j + 1]; ++k) y[ri[k]] += v[k] * xj;
  }
}

/* y += A' x  (per-column gather) */
static void csc_transpose_multiply_add(int32_t n, const int32_t* cs, const int32_t* ri,
                                       const double* v, const double* x, double* y) {
  for (int32_t j = 0; j < n; ++j) {
    double dot = 0.0;
    for (int32_t k = cs[j]; k < cs[j + 1]; ++k) dot += v[k] * x[ri[k]];
    y[j] += 1.0 * dot;
  }
}

/* primal step (src/pdhg/pdhg.cpp:393-400): x' = proj(x - tau (c + A'y)), x_bar = 2x' - x */
static void primal_step(int32_t n, double tau, const double* x, const double* cost,
                        const double* at_y, const double* lower, const double* upper,
                        double* x_next, double* extrapolated) {
  for (int32_t j = 0; j < n; ++j) {
    const double gradient = cost[j] + at_y[j];
    x_next[j] = project(x[j] - tau * gradient, lower[j], upper[j]);
    extrapolated[j] = 2.0 * x_next[j] - x[j];
  }
}

/* Exported single steps, so the known answers of the reference's GPU-slot tests
 * (tests/unit/test_gpu.cpp:107-177) can be checked against the code the solve runs. */
void oracle_csc_multiply(int32_t m, int32_t n, const int32_t* cs, const int32_t* ri,
                         const double* v, const double* x, double* y) {
  csc_multiply(m, n, cs, ri, v, x, y);
}

void oracle_csc_transpose_multiply(int32_t n, const int32_t* cs, const int32_t* ri,
                                   const double* v, const double* x, double* y) {
  for (int32_t j = 0; j < n; ++j) y[j] = 0.0;
  csc_transpose_multiply_add(n, cs, ri, v, x, y);
}

void oracle_primal_step(int32_t n, double tau, const double* x, const double* cost,
                        const double* at_y, const double* lower, const double* upper,
                        double* x_next, double* extrapolated) {
  primal_step(n, tau, x, cost, at_y, lower, upper, x_next, extrapolated);
}

/* ---- scaling: src/la/scaling.cpp:14-158 ----------------------------------------------- */

/* apply_pass (:14-40): the rebuild through add_entry + finalize(0.0) keeps the pattern and
 * the order, so it is an in-place product value * row_pass * column_pass. */
static void apply_pass(int32_t m, int32_t n, const int32_t* cs, const int32_t* ri, double* v,
                       const double* row_pass, const double* col_pass, double* row_scale,
                       double* col_scale) {
  for (int32_t j = 0; j < n; ++j) {
    const double cj = col_pass[j];
    for (int32_t k = cs[j]; k < cs[j + 1]; ++k) v[k] = v[k] * row_pass[ri[k]] * cj;
  }
  for (int32_t i = 0; i < m; ++i) row_scale[i] *= row_pass[i];
  for (int32_t j = 0; j < n; ++j) col_scale[j] *= col_pass[j];
}

int oracle_build_scaling(const oracle_lp* lp, const double* min_space_cost, int ruiz_iterations,
                         double* row_scale, double* col_scale, double* v, double* scaled_cost,
                         double* col_lower, double* col_upper, double* row_lower,
                         double* row_upper) {
  const int32_t m = lp->num_rows, n = lp->num_cols;
  const int32_t* cs = lp->col_starts;
  const int32_t* ri = lp->row_indices;
  double* row_acc = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
  double* col_acc = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double* row_pass = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
  double* col_pass = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  if (!row_acc || !col_acc || !row_pass || !col_pass) {
    free(row_acc); free(col_acc); free(row_pass); free(col_pass);
    return 1;
  }
  memcpy(v, lp->values, sizeof(double) * (size_t)lp->num_nonzeros);
  for (int32_t i = 0; i < m; ++i) row_scale[i] = 1.0;
  for (int32_t j = 0; j < n; ++j) col_scale[j] = 1.0;

  /* ruiz_round (:44-72) */
  for (int pass = 0; pass < ruiz_iterations; ++pass) {
    for (int32_t i = 0; i < m; ++i) row_acc[i] = 0.0;
    for (int32_t j = 0; j < n; ++j) col_acc[j] = 0.0;
    for (int32_t j = 0; j < n; ++j) {
      for (int32_t k = cs[j]; k < cs[j + 1]; ++k) {
        const double mag = fabs(v[k]);
        row_acc[ri[k]] = dmax(row_acc[ri[k]], mag);
        col_acc[j] = dmax(col_acc[j], mag);
      }
    }
    for (int32_t i = 0; i < m; ++i) row_pass[i] = row_acc[i] > 0.0 ? 1.0 / sqrt(row_acc[i]) : 1.0;
    for (int32_t j = 0; j < n; ++j) col_pass[j] = col_acc[j] > 0.0 ? 1.0 / sqrt(col_acc[j]) : 1.0;
    apply_pass(m, n, cs, ri, v, row_pass, col_pass, row_scale, col_scale);
  }

  /* pock_chambolle_round (:76-100), alpha = 1 */
  for (int32_t i = 0; i < m; ++i) row_acc[i] = 0.0;
  for (int32_t j = 0; j < n; ++j) col_acc[j] = 0.0;
  for (int32_t j = 0; j < n; ++j) {
    for (int32_t k = cs[j]; k < cs[j + 1]; ++k) {
      const double mag = fabs(v[k]);
      row_acc[ri[k]] += mag;
      col_acc[j] += mag;
    }
  }
  for (int32_t i = 0; i < m; ++i) row_pass[i] = row_acc[i] > 0.0 ? 1.0 / sqrt(row_acc[i]) : 1.0;
  for (int32_t j = 0; j < n; ++j) col_pass[j] = col_acc[j] > 0.0 ? 1.0 / sqrt(col_acc[j]) : 1.0;
  apply_pass(m, n, cs, ri, v, row_pass, col_pass, row_scale, col_scale);

  /* vectors (:127-145); scale_bound (:105-107) multiplies by 1/dc, it does not divide */
  for (int32_t j = 0; j < n; ++j) {
    const double dc = col_scale[j];
    scaled_cost[j] = min_space_cost[j] * dc;
    col_lower[j] = is_finite_bound(lp->col_lower[j]) ? lp->col_lower[j] * (1.0 / dc) : lp->col_lower[j];
    col_upper[j] = is_finite_bound(lp->col_upper[j]) ? lp->col_upper[j] * (1.0 / dc) : lp->col_upper[j];
  }
  for (int32_t i = 0; i < m; ++i) {
    const double dr = row_scale[i];
    row_lower[i] = is_finite_bound(lp->row_lower[i]) ? lp->row_lower[i] * dr : lp->row_lower[i];
    row_upper[i] = is_finite_bound(lp->row_upper[i]) ? lp->row_upper[i] * dr : lp->row_upper[i];
  }
  free(row_acc); free(col_acc); free(row_pass); free(col_pass);
  return 0;
}

/* src/la/scaling.cpp:161-194 */
double oracle_spectral_norm(int32_t m, int32_t n, const int32_t* cs, const int32_t* ri,
                            const double* val, int iterations, uint32_t seed) {
  if (m == 0 || n == 0 || cs[n] == 0) return 1.0;
  mt19937 g;
  mt_seed(&g, seed);
  double* v = (double*)malloc(sizeof(double) * (size_t)n);
  double* av = (double*)malloc(sizeof(double) * (size_t)m);
  if (!v || !av) { free(v); free(av); return 1.0; }
  for (int32_t j = 0; j < n; ++j) v[j] = (canonical(&g) * (1.0 - -1.0)) + -1.0;
  for (int32_t i = 0; i < m; ++i) av[i] = 0.0;
  double norm = 0.0;
  for (int step = 0; step < iterations; ++step) {
    double length = 0.0;
    for (int32_t j = 0; j < n; ++j) length += v[j] * v[j];
    length = sqrt(length);
    if (length == 0.0) { free(v); free(av); return 1.0; }
    for (int32_t j = 0; j < n; ++j) v[j] /= length;
    csc_multiply(m, n, cs, ri, val, v, av);
    for (int32_t j = 0; j < n; ++j) v[j] = 0.0;
    csc_transpose_multiply_add(n, cs, ri, val, av, v);
    double next = 0.0;
    for (int32_t j = 0; j < n; ++j) next += v[j] * v[j];
    norm = sqrt(sqrt(next));
  }
  free(v);
  free(av);
  return norm > 0.0 ? norm * 1.01 : 1.0;
}

/* ---- evaluate: src/pdhg/pdhg.cpp:143-263 ----------------------------------------------- */

typedef struct {
  const oracle_lp* lp;
  double* cost;       /* min-space cost (:287-291) */
  double bound_norm;  /* (:293-301) */
  double cost_norm;   /* (:292) */
} problem_t;

static oracle_residuals evaluate(const problem_t* p, const double* x, const double* y,
                                 double* activity, double* reduced) {
  const oracle_lp* lp = p->lp;
  const int32_t rows = lp->num_rows, cols = lp->num_cols;
  oracle_residuals r;
  memset(&r, 0, sizeof r);

  for (int32_t i = 0; i < rows; ++i) activity[i] = 0.0;
  if (rows > 0) csc_multiply(rows, cols, lp->col_starts, lp->row_indices, lp->values, x, activity);
  double primal_violation = 0.0;
  for (int32_t i = 0; i < rows; ++i) {
    const double a = activity[i];
    double violation = 0.0;
    if (is_finite_bound(lp->row_lower[i])) violation = dmax(violation, lp->row_lower[i] - a);
    if (is_finite_bound(lp->row_upper[i])) violation = dmax(violation, a - lp->row_upper[i]);
    primal_violation += violation * violation;
  }
  r.absolute_primal = sqrt(primal_violation);
  r.primal = r.absolute_primal / (1.0 + p->bound_norm);

  for (int32_t j = 0; j < cols; ++j) reduced[j] = p->cost[j];
  if (rows > 0) csc_transpose_multiply_add(cols, lp->col_starts, lp->row_indices, lp->values, y, reduced);

  double dual_violation = 0.0, bound_contribution = 0.0;
  for (int32_t j = 0; j < cols; ++j) {
    const double d = reduced[j];
    if (d > 0.0) {
      if (is_finite_bound(lp->col_lower[j])) bound_contribution += d * lp->col_lower[j];
      else dual_violation += d * d;
    } else if (d < 0.0) {
      if (is_finite_bound(lp->col_upper[j])) bound_contribution += d * lp->col_upper[j];
      else dual_violation += d * d;
    }
  }
  double support = 0.0;
  for (int32_t i = 0; i < rows; ++i) {
    const double yi = y[i];
    if (yi > 0.0) {
      if (is_finite_bound(lp->row_upper[i])) support += yi * lp->row_upper[i];
      else dual_violation += yi * yi;
    } else if (yi < 0.0) {
      if (is_finite_bound(lp->row_lower[i])) support += yi * lp->row_lower[i];
      else dual_violation += yi * yi;
    }
  }
  r.absolute_dual = sqrt(dual_violation);
  r.dual = r.absolute_dual / (1.0 + p->cost_norm);

  for (int32_t i = 0; i < rows; ++i) {
    if (lp->row_lower[i] == lp->row_upper[i]) continue;
    const double ls = is_finite_bound(lp->row_lower[i]) ? activity[i] - lp->row_lower[i] : INFINITY;
    const double us = is_finite_bound(lp->row_upper[i]) ? lp->row_upper[i] - activity[i] : INFINITY;
    r.complementarity = dmax(r.complementarity, fabs(y[i]) * dmin(ls, us));
  }
  for (int32_t j = 0; j < cols; ++j) {
    if (lp->col_lower[j] == lp->col_upper[j]) continue;
    const double ls = is_finite_bound(lp->col_lower[j]) ? x[j] - lp->col_lower[j] : INFINITY;
    const double us = is_finite_bound(lp->col_upper[j]) ? lp->col_upper[j] - x[j] : INFINITY;
    r.complementarity = dmax(r.complementarity, fabs(reduced[j]) * dmin(ls, us));
  }

  double primal_objective = 0.0;
  for (int32_t j = 0; j < cols; ++j) primal_objective += p->cost[j] * x[j];
  r.primal_objective = primal_objective;
  r.dual_objective = bound_contribution - support;
  const double absolute_gap = fabs(r.primal_objective - r.dual_objective);
  r.gap = absolute_gap / (1.0 + fabs(r.primal_objective) + fabs(r.dual_objective));
  r.gap_as_verified = absolute_gap / dmax(1.0, fabs(r.primal_objective));
  return r;
}

static double worst(const oracle_residuals* r) { return dmax(dmax(r->primal, r->dual), r->gap); }

/* :119-122 */
static int meets_request(const oracle_residuals* r, double tol) {
  return r->primal <= tol && r->dual <= tol && r->gap <= tol && r->absolute_primal <= 1e-7;
}
/* :127-131 */
static int meets_project_standard(const oracle_residuals* r) {
  return r->absolute_primal <= 1e-7 && r->absolute_dual <= 1e-7 && r->gap_as_verified <= 1e-9 &&
         r->complementarity <= 1e-6;
}

static void problem_init(problem_t* p, const oracle_lp* lp) {
  const double sense = lp->maximize ? -1.0 : 1.0;
  p->lp = lp;
  p->cost = (double*)malloc(sizeof(double) * (size_t)(lp->num_cols > 0 ? lp->num_cols : 1));
  double sq = 0.0;
  for (int32_t j = 0; j < lp->num_cols; ++j) {
    p->cost[j] = sense * lp->cost[j];
  }
  for (int32_t j = 0; j < lp->num_cols; ++j) sq += p->cost[j] * p->cost[j];
  p->cost_norm = sqrt(sq);
  double bs = 0.0;
  for (int32_t i = 0; i < lp->num_rows; ++i) {
    const double b = is_finite_bound(lp->row_lower[i])
                         ? lp->row_lower[i]
                         : (is_finite_bound(lp->row_upper[i]) ? lp->row_upper[i] : 0.0);
    bs += b * b;
  }
  p->bound_norm = sqrt(bs);
}

oracle_residuals oracle_evaluate(const oracle_lp* lp, const double* x, const double* y,
                                 double* activity, double* reduced) {
  problem_t p;
  problem_init(&p, lp);
  double* act = activity ? activity : (double*)malloc(sizeof(double) * (size_t)(lp->num_rows + 1));
  double* red = reduced ? reduced : (double*)malloc(sizeof(double) * (size_t)(lp->num_cols + 1));
  const oracle_residuals r = evaluate(&p, x, y, act, red);
  if (!activity) free(act);
  if (!reduced) free(red);
  free(p.cost);
  return r;
}

/* ---- solve_pdhg: src/pdhg/pdhg.cpp:267-726 ---------------------------------------------- */

#define ALLOC(T, count) ((T*)calloc((size_t)((count) > 0 ? (count) : 1), sizeof(T)))

int oracle_pdhg_solve(const oracle_lp* lp, double tolerance, int64_t iteration_option,
                      int use_restarts, int stop_at_request, int64_t random_seed,
                      double* col_value, double* row_dual_out, double* col_dual_out,
                      oracle_pdhg_out* out) {
  memset(out, 0, sizeof *out);
  const int32_t rows = lp->num_rows, cols = lp->num_cols;
  const int32_t* cs = lp->col_starts;
  const int32_t* ri = lp->row_indices;
  const double sense = lp->maximize ? -1.0 : 1.0;
  const size_t n = (size_t)cols, m = (size_t)rows;

  problem_t problem;
  problem_init(&problem, lp);

  /* preconditioning (:304-307) */
  double* row_scale = ALLOC(double, m);
  double* col_scale = ALLOC(double, n);
  double* sv = ALLOC(double, lp->num_nonzeros);
  double* s_cost = ALLOC(double, n);
  double* s_cl = ALLOC(double, n);
  double* s_cu = ALLOC(double, n);
  double* s_rl = ALLOC(double, m);
  double* s_ru = ALLOC(double, m);
  oracle_build_scaling(lp, problem.cost, 10, row_scale, col_scale, sv, s_cost, s_cl, s_cu, s_rl, s_ru);
  const double spectral_norm =
      oracle_spectral_norm(rows, cols, cs, ri, sv, 30, (uint32_t)random_seed + 1u);
  out->spectral_norm = spectral_norm;

  const int64_t iteration_limit = iteration_option < 0 ? 1000000 : iteration_option;

  double* x = ALLOC(double, n);
  double* y = ALLOC(double, m);
  for (int32_t j = 0; j < cols; ++j) x[j] = project(0.0, s_cl[j], s_cu[j]);
  double* x_next = ALLOC(double, n);
  double* y_next = ALLOC(double, m);
  double* extrapolated = ALLOC(double, n);
  double* at_y = ALLOC(double, n);
  double* a_x = ALLOC(double, m);
  double* x_sum = ALLOC(double, n);
  double* y_sum = ALLOC(double, m);
  int64_t averaged = 0;
  double* x_restart = ALLOC(double, n);
  double* y_restart = ALLOC(double, m);
  memcpy(x_restart, x, n * sizeof(double));
  memcpy(y_restart, y, m * sizeof(double));
  double* x_unscaled = ALLOC(double, n);
  double* y_unscaled = ALLOC(double, m);
  double* activity = ALLOC(double, m);
  double* reduced = ALLOC(double, n);
  double* cur_x = ALLOC(double, n);
  double* cur_y = ALLOC(double, m);
  double* avg_x = ALLOC(double, n);
  double* avg_y = ALLOC(double, m);
  double* dx = ALLOC(double, n);
  double* adx = ALLOC(double, m);
  double* best_x = ALLOC(double, n);
  double* best_y = ALLOC(double, m);
  memcpy(best_x, x, n * sizeof(double));
  memcpy(best_y, y, m * sizeof(double));

  double eta = spectral_norm > 0.0 ? 1.0 / spectral_norm : 1.0;
  double omega = 1.0;
  int64_t iteration = 0, restarts = 0, last_restart = 0, attempts = 0, evaluations = 0;
  double restart_kkt = INFINITY;
  oracle_residuals best;
  memset(&best, 0, sizeof best);
  best.primal = best.dual = best.gap = INFINITY;
  int converged = 0;

  for (;;) {
    if (iteration >= iteration_limit) break;
    ++attempts;
    const double tau = eta / omega;
    const double sigma = eta * omega;

    /* primal (:393-400) */
    for (int32_t j = 0; j < cols; ++j) at_y[j] = 0.0;
    if (rows > 0) csc_transpose_multiply_add(cols, cs, ri, sv, y, at_y);
    primal_step(cols, tau, x, s_cost, at_y, s_cl, s_cu, x_next, extrapolated);
    /* dual (:403-408) */
    if (rows > 0) csc_multiply(rows, cols, cs, ri, sv, extrapolated, a_x);
    for (int32_t i = 0; i < rows; ++i) {
      const double v = y[i] + sigma * a_x[i];
      y_next[i] = v - sigma * project(v / sigma, s_rl[i], s_ru[i]);
    }
    /* adaptive step (:413-496) */
    double movement = 0.0;
    for (int32_t j = 0; j < cols; ++j) {
      const double d = x_next[j] - x[j];
      movement += 0.5 * omega * d * d;
    }
    for (int32_t i = 0; i < rows; ++i) {
      const double d = y_next[i] - y[i];
      movement += 0.5 * d * d / omega;
    }
    double interaction = 0.0;
    if (rows > 0) {
      for (int32_t j = 0; j < cols; ++j) dx[j] = x_next[j] - x[j];
      csc_multiply(rows, cols, cs, ri, sv, dx, adx);
      for (int32_t i = 0; i < rows; ++i) interaction += (y_next[i] - y[i]) * adx[i];
      interaction = fabs(interaction);
    }
    const int no_information = interaction <= 0.0;
    const double limit = no_information ? INFINITY : movement / interaction;
    const double exponent = (double)(iteration + 1 > 2 ? iteration + 1 : 2);
    const double shrink = 1.0 - pow(exponent, -0.3);
    const double grow = 1.0 + pow(exponent, -0.6);
    const double proposed = dmin(shrink * limit, grow * eta);
    if (eta <= limit) {
      double* t = x; x = x_next; x_next = t;
      t = y; y = y_next; y_next = t;
      for (int32_t j = 0; j < cols; ++j) x_sum[j] += x[j];
      for (int32_t i = 0; i < rows; ++i) y_sum[i] += y[i];
      ++averaged;
      ++iteration;
    }
    const double eta_ceiling = 1.0e3 / dmax(spectral_norm, 1e-12);
    if (!no_information) eta = dclamp(proposed, 1e-12, eta_ceiling);

    /* convergence and restart (:502-643) */
    if (iteration == 0) continue;
    if (iteration % 40 != 0 && !no_information) continue;
    ++evaluations;

    for (int32_t j = 0; j < cols; ++j) x_unscaled[j] = x[j] * col_scale[j];
    for (int32_t i = 0; i < rows; ++i) y_unscaled[i] = y[i] * row_scale[i];
    memcpy(cur_x, x_unscaled, n * sizeof(double));
    memcpy(cur_y, y_unscaled, m * sizeof(double));
    const oracle_residuals current = evaluate(&problem, cur_x, cur_y, activity, reduced);
    const oracle_residuals* chosen = &current;
    const double* chosen_x = cur_x;
    const double* chosen_y = cur_y;
    oracle_residuals average;
    if (averaged > 0) {
      const double count = (double)averaged;
      for (int32_t j = 0; j < cols; ++j) avg_x[j] = x_sum[j] / count;
      for (int32_t i = 0; i < rows; ++i) avg_y[i] = y_sum[i] / count;
      for (int32_t j = 0; j < cols; ++j) avg_x[j] = avg_x[j] * col_scale[j];
      for (int32_t i = 0; i < rows; ++i) avg_y[i] = avg_y[i] * row_scale[i];
      average = evaluate(&problem, avg_x, avg_y, activity, reduced);
      if (worst(&average) < worst(&current)) {
        chosen = &average;
        chosen_x = avg_x;
        chosen_y = avg_y;
      }
    }
    const oracle_residuals better = *chosen;
    if (worst(&better) < worst(&best)) {
      best = better;
      memcpy(best_x, chosen_x, n * sizeof(double));
      memcpy(best_y, chosen_y, m * sizeof(double));
    }
    const int stop_here =
        meets_request(&better, tolerance) && (stop_at_request || meets_project_standard(&better));
    if (stop_here) {
      best = better;
      memcpy(best_x, chosen_x, n * sizeof(double));
      memcpy(best_y, chosen_y, m * sizeof(double));
      converged = 1;
      break;
    }
    if (use_restarts) {
      const double kkt = worst(&better);
      const int64_t since = iteration - last_restart;
      const int sufficient = kkt <= 0.2 * restart_kkt;
      const int64_t art = (int64_t)(0.36 * (double)iteration);
      const int artificial = since >= (art > 40 ? art : 40);
      if (sufficient || artificial) {
        double dxs = 0.0, dys = 0.0;
        for (int32_t j = 0; j < cols; ++j) {
          const double d = x[j] - x_restart[j];
          dxs += d * d;
        }
        for (int32_t i = 0; i < rows; ++i) {
          const double d = y[i] - y_restart[i];
          dys += d * d;
        }
        const double dx_norm = sqrt(dxs), dy_norm = sqrt(dys);
        if (dx_norm > 1e-12 && dy_norm > 1e-12) {
          const double theta = 0.5;
          omega = exp(theta * log(dy_norm / dx_norm) + (1.0 - theta) * log(omega));
          omega = dclamp(omega, 1e-6, 1e6);
        }
        memset(x_sum, 0, n * sizeof(double));
        memset(y_sum, 0, m * sizeof(double));
        averaged = 0;
        memcpy(x_restart, x, n * sizeof(double));
        memcpy(y_restart, y, m * sizeof(double));
        restart_kkt = kkt;
        last_restart = iteration;
        ++restarts;
      }
    }
  }

  /* report (:647-716) */
  const oracle_residuals fin = evaluate(&problem, best_x, best_y, activity, reduced);
  if (col_value) memcpy(col_value, best_x, n * sizeof(double));
  if (col_dual_out) for (int32_t j = 0; j < cols; ++j) col_dual_out[j] = sense * reduced[j];
  if (row_dual_out) for (int32_t i = 0; i < rows; ++i) row_dual_out[i] = sense * (-best_y[i]);
  const int verifiable = converged && meets_project_standard(&fin);
  out->status = verifiable ? ORACLE_OPTIMAL : (converged ? ORACLE_FEASIBLE : ORACLE_ITERATION_LIMIT);
  out->converged = converged;
  out->iterations = iteration;
  out->attempts = attempts;
  out->restarts = restarts;
  out->evaluations = evaluations;
  out->final_eta = eta;
  out->final_omega = omega;
  out->final_residuals = fin;
  /* Model::evaluate_objective (src/core/model.cpp:99-105): starts from the offset */
  double obj = lp->objective_offset;
  for (int32_t j = 0; j < cols; ++j) obj += lp->cost[j] * best_x[j];
  out->objective = obj;
  out->dual_bound = verifiable ? sense * fin.dual_objective + lp->objective_offset
                               : (lp->maximize ? INFINITY : -INFINITY);

  free(problem.cost);
  free(row_scale); free(col_scale); free(sv); free(s_cost); free(s_cl); free(s_cu);
  free(s_rl); free(s_ru); free(x); free(y); free(x_next); free(y_next); free(extrapolated);
  free(at_y); free(a_x); free(x_sum); free(y_sum); free(x_restart); free(y_restart);
  free(x_unscaled); free(y_unscaled); free(activity); free(reduced); free(cur_x); free(cur_y);
  free(avg_x); free(avg_y); free(dx); free(adx); free(best_x); free(best_y);
  return 0;
}
