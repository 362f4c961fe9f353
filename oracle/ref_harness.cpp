// TEST INFRASTRUCTURE ONLY -- never linked into the product.
//
// A C entry point over the reference solver's own restarted-PDHG path, so that the tests and
// the CPU arm of bench.py can run the UNMODIFIED reference code on the same inputs as the
// CUDA path. This file is ours; the sources it links are compiled in place from the
// reference tree by oracle/Makefile (target `ref`), and the result lands in oracle/_ref/.
//
// What it binds (reference file:line):
//   sankhya::pdhg::solve_pdhg            src/pdhg/pdhg.cpp:267      include/sankhya/pdhg.hpp:15
//   sankhya::build_scaling               src/la/scaling.cpp:111     src/la/scaling.hpp:65
//   sankhya::estimate_spectral_norm      src/la/scaling.cpp:161     src/la/scaling.hpp:72
//   sankhya::farkas_proves_infeasible    src/core/certificate.cpp:29
//   sankhya::ray_proves_unbounded        src/core/certificate.cpp:121
//   sankhya::io::read_model              include/sankhya/io.hpp:53  (MPS/LP files, for pins)
//   sankhya::qp::solve_convex_qp         src/qp/qp_condat_vu.cpp:150 include/sankhya/qp.hpp:20
//   sankhya::Solution::recompute_quality src/core/model.cpp:228      include/sankhya/model.hpp:373
//   sankhya::ipm::solve_ipm (warm start) src/ipm/ipm.cpp            include/sankhya/ipm.hpp:41,
//     inside a restatement of its caller polish_with_the_interior_point
//     (src/core/solve.cpp:184-243), which sits among the whole solve() machinery
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "sankhya/certificate.hpp"
#include "sankhya/io.hpp"
#include "sankhya/ipm.hpp"
#include "sankhya/logging.hpp"
#include "sankhya/model.hpp"
#include "sankhya/options.hpp"
#include "sankhya/pdhg.hpp"
#include "sankhya/qp.hpp"

#include "la/scaling.hpp"

extern "C" {

/// One LP in the reference's own storage convention: CSC with ascending rows per column,
/// int32 indices, FP64 values, absent bounds as +-inf.
struct ref_lp {
  std::int32_t num_rows;
  std::int32_t num_cols;
  std::int32_t num_nonzeros;
  const std::int32_t* col_starts;
  const std::int32_t* row_indices;
  const double* values;
  const double* cost;
  const double* col_lower;
  const double* col_upper;
  const double* row_lower;
  const double* row_upper;
  std::int32_t maximize;
  double objective_offset;
};

struct ref_pdhg_out {
  std::int32_t status;  // sankhya::SolveStatus numeric value
  std::int64_t iterations;
  double objective;
  double dual_bound;
  double solve_seconds;
  double primal_infeasibility;
  double dual_infeasibility;
  char algorithm[32];
  char message[1024];
};

}  // extern "C"

namespace {

sankhya::Model to_model(const ref_lp& lp) {
  using namespace sankhya;
  Model model;
  model.sense = lp.maximize ? ObjSense::kMaximize : ObjSense::kMinimize;
  model.objective_offset = lp.objective_offset;
  const auto n = static_cast<std::size_t>(lp.num_cols);
  const auto m = static_cast<std::size_t>(lp.num_rows);
  model.col_cost.assign(lp.cost, lp.cost + n);
  model.col_lower.assign(lp.col_lower, lp.col_lower + n);
  model.col_upper.assign(lp.col_upper, lp.col_upper + n);
  model.col_type.assign(n, VarType::kContinuous);
  model.row_lower.assign(lp.row_lower, lp.row_lower + m);
  model.row_upper.assign(lp.row_upper, lp.row_upper + m);
  model.matrix.reset(lp.num_rows, lp.num_cols);
  model.matrix.reserve(static_cast<std::size_t>(lp.num_nonzeros));
  for (Index j = 0; j < lp.num_cols; ++j) {
    for (Index k = lp.col_starts[j]; k < lp.col_starts[j + 1]; ++k) {
      model.matrix.add_entry(lp.row_indices[k], j, lp.values[k]);
    }
  }
  // Drop tolerance 0: the caller's matrix is taken exactly as given, so the CUDA path and
  // this one see the same entries.
  model.matrix.finalize(0.0);
  return model;
}

void copy_text(char* dst, std::size_t cap, const std::string& text) {
  if (cap == 0) return;
  const std::size_t len = std::min(cap - 1, text.size());
  std::memcpy(dst, text.data(), len);
  dst[len] = '\0';
}

}  // namespace

extern "C" {

/// Runs sankhya::pdhg::solve_pdhg with the named options; outputs may be NULL.
int ref_pdhg_solve(const ref_lp* lp, double tolerance, std::int64_t iteration_limit,
                   double time_limit, int restart, int stop_at_request, std::int64_t seed,
                   int log_level, double* col_value, double* row_dual, double* col_dual,
                   ref_pdhg_out* out) {
  using namespace sankhya;
  try {
    const Model model = to_model(*lp);
    Options options;
    options.set_double("pdhg_tolerance", tolerance);
    options.set_int("iteration_limit", iteration_limit);
    if (time_limit > 0.0 && time_limit < std::numeric_limits<double>::infinity()) {
      options.set_double("time_limit", time_limit);
    }
    options.set_bool("pdhg_restart", restart != 0);
    options.set_bool("pdhg_stop_at_request", stop_at_request != 0);
    options.set_int("random_seed", seed);
    Logger logger(stdout, static_cast<LogLevel>(log_level));
    const Solution s = pdhg::solve_pdhg(model, options, logger);
    std::fflush(stdout);
    out->status = static_cast<std::int32_t>(s.status);
    out->iterations = s.iterations;
    out->objective = s.objective;
    out->dual_bound = s.dual_bound;
    out->solve_seconds = s.solve_seconds;
    out->primal_infeasibility = s.primal_infeasibility;
    out->dual_infeasibility = s.dual_infeasibility;
    copy_text(out->algorithm, sizeof(out->algorithm), s.algorithm);
    copy_text(out->message, sizeof(out->message), s.message);
    const auto n = static_cast<std::size_t>(lp->num_cols);
    const auto m = static_cast<std::size_t>(lp->num_rows);
    if (col_value && s.col_value.size() == n) std::memcpy(col_value, s.col_value.data(), n * 8);
    if (col_dual && s.col_dual.size() == n) std::memcpy(col_dual, s.col_dual.data(), n * 8);
    if (row_dual && s.row_dual.size() == m) std::memcpy(row_dual, s.row_dual.data(), m * 8);
    return 0;
  } catch (const std::exception& e) {
    copy_text(out->message, sizeof(out->message), e.what());
    return 1;
  }
}

/// sankhya::build_scaling on the min-space cost (sense folded in by the caller).
/// Writes Dr[m], Dc[n], the scaled values[nnz] (CSC order) and the scaled vectors.
int ref_build_scaling(const ref_lp* lp, const double* min_space_cost, int ruiz_iterations,
                      double* row_scale, double* col_scale, double* scaled_values,
                      double* scaled_cost, double* col_lower, double* col_upper,
                      double* row_lower, double* row_upper) {
  using namespace sankhya;
  try {
    const Model model = to_model(*lp);
    const std::vector<double> cost(min_space_cost, min_space_cost + lp->num_cols);
    const Scaling s = build_scaling(model, cost, ruiz_iterations);
    const auto n = static_cast<std::size_t>(lp->num_cols);
    const auto m = static_cast<std::size_t>(lp->num_rows);
    std::memcpy(row_scale, s.row.data(), m * 8);
    std::memcpy(col_scale, s.column.data(), n * 8);
    std::memcpy(scaled_values, s.matrix.values().data(), s.matrix.values().size() * 8);
    std::memcpy(scaled_cost, s.cost.data(), n * 8);
    std::memcpy(col_lower, s.col_lower.data(), n * 8);
    std::memcpy(col_upper, s.col_upper.data(), n * 8);
    std::memcpy(row_lower, s.row_lower.data(), m * 8);
    std::memcpy(row_upper, s.row_upper.data(), m * 8);
    return 0;
  } catch (...) {
    return 1;
  }
}

/// sankhya::estimate_spectral_norm on the given CSC matrix.
double ref_spectral_norm(const ref_lp* lp, int iterations, unsigned seed) {
  const sankhya::Model model = to_model(*lp);
  return sankhya::estimate_spectral_norm(model.matrix, iterations, seed);
}

/// sankhya::farkas_proves_infeasible / ray_proves_unbounded. Returns 1 when the certificate
/// proves its verdict, 0 when it does not (with the reason), -1 on an internal error.
/// The reference's Model::validate (src/core/model.cpp:125-210) of the LP: returns 1 when it
/// passes, else 0 with validate()'s text in `why` -- the text solve_pdhg reports as its
/// kModelError message (src/pdhg/pdhg.cpp:273-278).
int ref_validate(const ref_lp* lp, char* why, int why_len) {
  const std::string text = to_model(*lp).validate();
  copy_text(why, static_cast<std::size_t>(why_len), text);
  return text.empty() ? 1 : 0;
}

int ref_farkas_check(const ref_lp* lp, const double* y, char* why, int why_len) {
  try {
    const sankhya::Model model = to_model(*lp);
    std::string reason;
    const std::vector<double> v(y, y + lp->num_rows);
    const bool ok = sankhya::farkas_proves_infeasible(model, v, &reason);
    if (why) copy_text(why, static_cast<std::size_t>(why_len), reason);
    return ok ? 1 : 0;
  } catch (...) {
    return -1;
  }
}

int ref_ray_check(const ref_lp* lp, const double* d, char* why, int why_len) {
  try {
    const sankhya::Model model = to_model(*lp);
    std::string reason;
    const std::vector<double> v(d, d + lp->num_cols);
    const bool ok = sankhya::ray_proves_unbounded(model, v, &reason);
    if (why) copy_text(why, static_cast<std::size_t>(why_len), reason);
    return ok ? 1 : 0;
  } catch (...) {
    return -1;
  }
}

/// Reads an MPS/LP file with the reference reader. Call once with NULL arrays to get the
/// sizes in *lp (num_rows, num_cols, num_nonzeros), then again with arrays of those sizes.
/// The caller owns every array; lp's pointer members are cast away from const to fill them.
int ref_read_model(const char* path, ref_lp* lp, char* why, int why_len) {
  using namespace sankhya;
  try {
    Model model;
    const io::ReadResult read = io::read_model(path, &model);
    if (!read.ok) {
      if (why) copy_text(why, static_cast<std::size_t>(why_len), read.error);
      return 1;
    }
    if (lp->col_starts == nullptr) {
      lp->num_rows = model.num_rows();
      lp->num_cols = model.num_cols();
      lp->num_nonzeros = model.num_nonzeros();
      lp->maximize = model.sense == ObjSense::kMaximize ? 1 : 0;
      lp->objective_offset = model.objective_offset;
      return 0;
    }
    const auto n = static_cast<std::size_t>(model.num_cols());
    const auto m = static_cast<std::size_t>(model.num_rows());
    const auto& cs = model.matrix.column_starts();
    std::memcpy(const_cast<std::int32_t*>(lp->col_starts), cs.data(), (n + 1) * 4);
    std::memcpy(const_cast<std::int32_t*>(lp->row_indices), model.matrix.row_indices().data(),
                model.matrix.row_indices().size() * 4);
    std::memcpy(const_cast<double*>(lp->values), model.matrix.values().data(),
                model.matrix.values().size() * 8);
    std::memcpy(const_cast<double*>(lp->cost), model.col_cost.data(), n * 8);
    std::memcpy(const_cast<double*>(lp->col_lower), model.col_lower.data(), n * 8);
    std::memcpy(const_cast<double*>(lp->col_upper), model.col_upper.data(), n * 8);
    std::memcpy(const_cast<double*>(lp->row_lower), model.row_lower.data(), m * 8);
    std::memcpy(const_cast<double*>(lp->row_upper), model.row_upper.data(), m * 8);
    return 0;
  } catch (const std::exception& e) {
    if (why) copy_text(why, static_cast<std::size_t>(why_len), e.what());
    return 1;
  }
}

}  // extern "C"

extern "C" {

/// sankhya::qp::solve_convex_qp on the LP plus a Hessian given as its lower triangle in CSC
/// (the reference's Model::hessian storage). Outputs may be NULL.
int ref_qp_solve(const ref_lp* lp, const std::int32_t* h_col_starts,
                 const std::int32_t* h_row_indices, const double* h_values, double tolerance,
                 std::int64_t iteration_limit, double* col_value, double* row_dual,
                 double* col_dual, ref_pdhg_out* out) {
  using namespace sankhya;
  try {
    Model model = to_model(*lp);
    model.hessian.reset(lp->num_cols, lp->num_cols);
    for (Index j = 0; j < lp->num_cols; ++j) {
      for (Index k = h_col_starts[j]; k < h_col_starts[j + 1]; ++k) {
        model.hessian.add_entry(h_row_indices[k], j, h_values[k]);
      }
    }
    model.hessian.finalize(0.0);
    Options options;
    options.set_double("qp_tolerance", tolerance);
    options.set_int("iteration_limit", iteration_limit);
    Logger logger(stdout, LogLevel::kOff);
    const Solution s = qp::solve_convex_qp(model, options, logger);
    out->status = static_cast<std::int32_t>(s.status);
    out->iterations = s.iterations;
    out->objective = s.objective;
    out->dual_bound = s.dual_bound;
    out->solve_seconds = s.solve_seconds;
    out->primal_infeasibility = s.primal_infeasibility;
    out->dual_infeasibility = s.dual_infeasibility;
    copy_text(out->algorithm, sizeof(out->algorithm), s.algorithm);
    copy_text(out->message, sizeof(out->message), s.message);
    const auto n = static_cast<std::size_t>(lp->num_cols);
    const auto m = static_cast<std::size_t>(lp->num_rows);
    if (col_value && s.col_value.size() == n) std::memcpy(col_value, s.col_value.data(), n * 8);
    if (col_dual && s.col_dual.size() == n) std::memcpy(col_dual, s.col_dual.data(), n * 8);
    if (row_dual && s.row_dual.size() == m) std::memcpy(row_dual, s.row_dual.data(), m * 8);
    return 0;
  } catch (const std::exception& e) {
    copy_text(out->message, sizeof(out->message), e.what());
    return 1;
  }
}

}  // extern "C"

extern "C" {

/// Solution::recompute_quality of a given point (x, row_dual, col_dual in the reference's
/// sign conventions) and dual bound on the LP. out[8] = primal_infeasibility,
/// primal_infeasibility_scaled, dual_infeasibility, dual_infeasibility_scaled,
/// complementarity_violation, objective, absolute_gap, relative_gap.
int ref_recompute_quality(const ref_lp* lp, const double* col_value, const double* row_dual,
                          const double* col_dual, double dual_bound, double* out) {
  using namespace sankhya;
  try {
    const Model model = to_model(*lp);
    Solution s;
    s.allocate_for(model);
    const auto n = static_cast<std::size_t>(lp->num_cols);
    const auto m = static_cast<std::size_t>(lp->num_rows);
    std::copy(col_value, col_value + n, s.col_value.begin());
    std::copy(col_dual, col_dual + n, s.col_dual.begin());
    std::copy(row_dual, row_dual + m, s.row_dual.begin());
    s.dual_bound = dual_bound;
    s.recompute_quality(model);
    out[0] = s.primal_infeasibility;
    out[1] = s.primal_infeasibility_scaled;
    out[2] = s.dual_infeasibility;
    out[3] = s.dual_infeasibility_scaled;
    out[4] = s.complementarity_violation;
    out[5] = s.objective;
    out[6] = s.absolute_gap;
    out[7] = s.relative_gap;
    return 0;
  } catch (const std::exception&) {
    return 1;
  }
}

}  // extern "C"

// ---- the interior-point polish of a first-order answer ------------------------------------
//
// polish_with_the_interior_point (src/core/solve.cpp:184-243) runs right after the PDHG
// engine at the call site the GPU library replaces (src/core/solve.cpp:392-393). This entry
// point repeats its few steps -- the options it sets, the warm start it builds, the "better"
// rule and the "+ipm" algorithm name -- around the reference's own interior point.
extern "C" {

struct ref_polish_out {
  std::int32_t status;    // sankhya::SolveStatus of the merged answer
  std::int32_t polished;  // 1 when the interior point's answer replaced the first one
  std::int64_t iterations;
  std::int64_t polish_iterations;
  double objective;
  double primal_infeasibility;
  double dual_infeasibility;
  char algorithm[64];
  char message[1024];
};

/// first_status is the first answer's sankhya::SolveStatus value; first_algorithm its
/// Solution::algorithm (e.g. "pdhg-gpu"); first_scaled_worst its max(primal, dual)
/// infeasibility over the recompute_quality scales; first_message its Solution::message (may
/// be NULL). col_value / row_dual / col_dual are the first answer in the reference's units and
/// signs; polished outputs may be NULL.
int ref_polish_ipm(const ref_lp* lp, const double* col_value, const double* row_dual,
                   const double* col_dual, std::int32_t first_status, std::int64_t first_iterations,
                   const char* first_algorithm, double first_scaled_worst, double* x_out,
                   double* rd_out, double* cd_out, ref_polish_out* out,
                   const char* first_message) {
  using namespace sankhya;
  try {
    const Model model = to_model(*lp);
    const auto n = static_cast<std::size_t>(lp->num_cols);
    const auto m = static_cast<std::size_t>(lp->num_rows);
    Options options;
    // solve.cpp:196-214: the polish's own iteration cap and clock
    Options polish = options;
    polish.set_int("iteration_limit", options.get_int("polish_iteration_limit"));
    polish.set_double("time_limit", options.get_double("polish_max_seconds"));
    Logger logger(stdout, LogLevel::kWarning);
    const ipm::WarmStart warm{std::vector<double>(col_value, col_value + n),
                              std::vector<double>(row_dual, row_dual + m),
                              std::vector<double>(col_dual, col_dual + n)};
    Solution polished = ipm::solve_ipm(model, polish, logger, &warm);
    // solve.cpp:218-231: kept only when better
    const double worst = std::max(polished.primal_infeasibility_scaled,
                                  polished.dual_infeasibility_scaled);
    const bool better = polished.status == SolveStatus::kOptimal ||
                        (polished.status == SolveStatus::kFeasible && worst < first_scaled_worst);
    out->polished = better ? 1 : 0;
    out->polish_iterations = polished.iterations;
    std::string algorithm = first_algorithm ? first_algorithm : "";
    // solve.cpp:225-241: the merged message of the answer that stands
    std::string message = first_message ? first_message : "";
    if (better) {
      message += "; polished by the interior point in " + std::to_string(polished.iterations) +
                 " iterations" + (polished.message.empty() ? std::string()
                                                           : " (" + polished.message + ")");
    } else {
      message += "; the interior-point polish did not improve it (" +
                 std::string(to_string(polished.status)) + " after " +
                 std::to_string(polished.iterations) + " iterations: " + polished.message + ")";
    }
    if (better) {
      algorithm += "+ipm";  // solve.cpp:237
      out->status = static_cast<std::int32_t>(polished.status);
      out->iterations = polished.iterations + first_iterations;
      out->objective = polished.objective;
      out->primal_infeasibility = polished.primal_infeasibility;
      out->dual_infeasibility = polished.dual_infeasibility;
      if (x_out && polished.col_value.size() == n) std::memcpy(x_out, polished.col_value.data(), n * 8);
      if (rd_out && polished.row_dual.size() == m) std::memcpy(rd_out, polished.row_dual.data(), m * 8);
      if (cd_out && polished.col_dual.size() == n) std::memcpy(cd_out, polished.col_dual.data(), n * 8);
    } else {
      out->status = first_status;
      out->iterations = first_iterations;
    }
    std::snprintf(out->algorithm, sizeof out->algorithm, "%s", algorithm.c_str());
    std::snprintf(out->message, sizeof out->message, "%s", message.c_str());
    return 0;
  } catch (const std::exception& e) {
    std::snprintf(out->message, sizeof out->message, "%s", e.what());
    return 1;
  }
}

}  // extern "C"
