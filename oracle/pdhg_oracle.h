/* TEST INFRASTRUCTURE ONLY -- the oracle. Never linked into the product library.
 *
 * A plain-C, FP64, single-threaded restatement of the reference solver's restarted-PDHG
 * path, written operation for operation in the reference's order so that on the same input
 * it reproduces the reference's iterates bit for bit (pinned against the reference build in
 * tests/test_oracle_pins.py). Every function cites the reference file:line it restates.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this. */
#ifndef SIH26_PDHG_ORACLE_H
#define SIH26_PDHG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One LP: CSC with ascending rows per column (include/sankhya/sparse.hpp:109-112), int32
 * indices, FP64 values; an absent bound is any |v| >= 1e30 (include/sankhya/types.hpp:32). */
typedef struct oracle_lp {
  int32_t num_rows;
  int32_t num_cols;
  int32_t num_nonzeros;
  const int32_t* col_starts;
  const int32_t* row_indices;
  const double* values;
  const double* cost;
  const double* col_lower;
  const double* col_upper;
  const double* row_lower;
  const double* row_upper;
  int32_t maximize;
  double objective_offset;
} oracle_lp;

/* The unscaled residual block of src/pdhg/pdhg.cpp:81-132. */
typedef struct oracle_residuals {
  double primal, dual, gap;
  double primal_objective, dual_objective;
  double absolute_primal, absolute_dual, gap_as_verified, complementarity;
} oracle_residuals;

/* Status values follow sankhya::SolveStatus (include/sankhya/model.hpp:62-80). */
enum {
  ORACLE_NOT_SOLVED = 0,
  ORACLE_OPTIMAL = 1,
  ORACLE_FEASIBLE = 5,
  ORACLE_ITERATION_LIMIT = 6,
  ORACLE_TIME_LIMIT = 7,
  ORACLE_MODEL_ERROR = 10
};

typedef struct oracle_pdhg_out {
  int32_t status;
  int32_t converged;
  int64_t iterations;   /* accepted iterations */
  int64_t attempts;     /* accepted + rejected steps */
  int64_t restarts;
  int64_t evaluations;
  double spectral_norm;
  double final_eta;
  double final_omega;
  double objective;     /* original sense, offset included */
  double dual_bound;
  oracle_residuals final_residuals;
} oracle_pdhg_out;

/* mt19937 + std::uniform_real_distribution<double>(lo, hi), as libstdc++ draws it. */
void oracle_uniform_draws(uint32_t seed, double lo, double hi, int64_t count, double* out);

/* src/la/scaling.cpp:111-158. */
int oracle_build_scaling(const oracle_lp* lp, const double* min_space_cost, int ruiz_iterations,
                         double* row_scale, double* col_scale, double* scaled_values,
                         double* scaled_cost, double* col_lower, double* col_upper,
                         double* row_lower, double* row_upper);

/* src/la/scaling.cpp:161-194, on the matrix (col_starts, row_indices, values). */
double oracle_spectral_norm(int32_t num_rows, int32_t num_cols, const int32_t* col_starts,
                            const int32_t* row_indices, const double* values, int iterations,
                            uint32_t seed);

/* The CSC products of src/la/sparse.cpp:202-229 (y = A x; y = A' x, y zeroed first) and the
 * primal step of src/pdhg/pdhg.cpp:393-400, as the solve below runs them. */
void oracle_csc_multiply(int32_t num_rows, int32_t num_cols, const int32_t* col_starts,
                         const int32_t* row_indices, const double* values, const double* x,
                         double* y);
void oracle_csc_transpose_multiply(int32_t num_cols, const int32_t* col_starts,
                                   const int32_t* row_indices, const double* values,
                                   const double* x, double* y);
void oracle_primal_step(int32_t n, double tau, const double* x, const double* cost,
                        const double* at_y, const double* lower, const double* upper,
                        double* x_next, double* extrapolated);

/* src/pdhg/pdhg.cpp:143-263: unscaled residuals of (x, y) in PDHG sign (y = -multiplier),
 * min-space cost. activity[m] and reduced[n] are outputs (may be NULL). */
oracle_residuals oracle_evaluate(const oracle_lp* lp, const double* x, const double* y,
                                 double* activity, double* reduced);

/* src/pdhg/pdhg.cpp:267-726 (time limit excluded: the oracle runs to its iteration limit).
 * Outputs follow pdhg.cpp:647-661: col_value[n], row_dual[m] = sense*(-y),
 * col_dual[n] = sense*(c+A'y). Any output pointer may be NULL. */
int oracle_pdhg_solve(const oracle_lp* lp, double tolerance, int64_t iteration_limit,
                      int restart, int stop_at_request, int64_t random_seed, double* col_value,
                      double* row_dual, double* col_dual, oracle_pdhg_out* out);

#ifdef __cplusplus
}
#endif

#endif
