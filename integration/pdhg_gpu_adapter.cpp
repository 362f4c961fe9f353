// The reference-side adapter: the one translation unit a maintainer adds to the SANKHYA solver
// (as src/gpu/pdhg_gpu_adapter.cpp, compiled when the GPU backend is enabled) so that
// run_lp_engine (src/core/solve.cpp:385-395) can call the GPU engine where it calls
// pdhg::solve_pdhg (include/sankhya/pdhg.hpp:15), and the QP path where it calls
// qp::solve_convex_qp (include/sankhya/qp.hpp:20). It turns the reference's Model and Options
// into the C-ABI structs of include/sankhya_pdhg_gpu.h and each result back into a Solution,
// using only the reference's own types and that header.
//
// Options: the PDHG rows the reference already has are read as they are. The GPU rows
// (pdhg_precision, pdhg_stop_rule, pdhg_detect_infeasibility, pdhg_mixed_switch_tolerance)
// are read only when the registry holds them (Options::exists): the reference's typed
// accessors abort on an unknown name, so the adapter works both before and after those rows
// are added, with the library's defaults until then.
#include <string>
#include <vector>

#include "sankhya/logging.hpp"
#include "sankhya/model.hpp"
#include "sankhya/options.hpp"
#include "sankhya_pdhg_gpu.h"

namespace sankhya::pdhg {

namespace {

SolveStatus to_solve_status(int32_t status) {
  // the values of sankhya_solve_status (include/sankhya/sankhya.h:53-66)
  switch (status) {
    case SANKHYA_PDHG_OPTIMAL: return SolveStatus::kOptimal;
    case SANKHYA_PDHG_FEASIBLE: return SolveStatus::kFeasible;
    case SANKHYA_PDHG_INFEASIBLE: return SolveStatus::kInfeasible;
    case SANKHYA_PDHG_UNBOUNDED: return SolveStatus::kUnbounded;
    case SANKHYA_PDHG_INFEASIBLE_OR_UNBOUNDED: return SolveStatus::kInfeasibleOrUnbounded;
    case SANKHYA_PDHG_ITERATION_LIMIT: return SolveStatus::kIterationLimit;
    case SANKHYA_PDHG_TIME_LIMIT: return SolveStatus::kTimeLimit;
    case SANKHYA_PDHG_NUMERICAL_ERROR: return SolveStatus::kNumericalError;
    case SANKHYA_PDHG_MODEL_ERROR: return SolveStatus::kModelError;
    default: return SolveStatus::kNotSolved;
  }
}

// The model as the ABI reads it: pointers into the frozen CSC (sparse.hpp:109-112) and the
// model's own vectors; nothing is copied.
sankhya_pdhg_problem problem_view(const Model& model) {
  const SparseMatrix& a = model.matrix;
  return sankhya_pdhg_problem{model.num_rows(), model.num_cols(), model.num_nonzeros(),
                              a.column_starts().data(), a.row_indices().data(),
                              a.values().data(), model.col_cost.data(), model.col_lower.data(),
                              model.col_upper.data(), model.row_lower.data(),
                              model.row_upper.data(), model.sense == ObjSense::kMaximize,
                              model.objective_offset};
}

sankhya_pdhg_params params_from(const Options& options) {
  sankhya_pdhg_params q;
  sankhya_pdhg_gpu_default_params(&q);
  q.tolerance = options.get_double("pdhg_tolerance");
  q.iteration_limit = options.get_int("iteration_limit");
  q.time_limit = options.get_double("time_limit");
  q.restart = options.get_bool("pdhg_restart");
  q.stop_at_request = options.get_bool("pdhg_stop_at_request");
  q.random_seed = options.get_int("random_seed");
  if (Options::exists("pdhg_precision"))
    q.precision = options.get_string("pdhg_precision") == "mixed" ? SANKHYA_PDHG_MIXED
                                                                 : SANKHYA_PDHG_FP64;
  if (Options::exists("pdhg_stop_rule"))
    q.stop_rule = options.get_string("pdhg_stop_rule") == "relative_kkt"
                      ? SANKHYA_PDHG_STOP_RELATIVE_KKT
                      : SANKHYA_PDHG_STOP_REFERENCE;
  if (Options::exists("pdhg_detect_infeasibility"))
    q.detect_infeasibility = options.get_bool("pdhg_detect_infeasibility") ? 1 : 0;
  if (Options::exists("pdhg_mixed_switch_tolerance"))
    q.mixed_switch_tolerance = options.get_double("pdhg_mixed_switch_tolerance");
  return q;
}

// One call's Solution and the certificate buffers the result writes into.
struct Pending {
  Solution s;
  std::vector<double> farkas, ray;
  sankhya_pdhg_result r{};
};

void bind(Pending& p, const Model& model, const char* algorithm) {
  p.s.allocate_for(model);
  p.s.algorithm = algorithm;                     // verify.cpp:85-89 looks for "gpu"
  p.farkas.assign(model.num_rows(), 0.0);
  p.ray.assign(model.num_cols(), 0.0);
  p.r.col_value = p.s.col_value.data();
  p.r.row_dual = p.s.row_dual.data();
  p.r.col_dual = p.s.col_dual.data();
  p.r.farkas_dual = p.farkas.data();             // filled when the status is INFEASIBLE
  p.r.primal_ray = p.ray.data();                 // filled when a ray is reported
}

// no CPU fallback: the failure is the answer
Solution failed(Pending& p, const char* engine) {
  p.s.status = SolveStatus::kNumericalError;
  p.s.message = std::string(engine) + ": " + sankhya_pdhg_gpu_last_error();
  return std::move(p.s);
}

// measured_here: recompute the quality block on the host (recompute_quality, as
// pdhg.cpp:716 does); otherwise take the block the device measured, term for term the same.
Solution finish(Pending& p, const Model& model, bool measured_here) {
  Solution& s = p.s;
  s.status = to_solve_status(p.r.status);
  if (s.status == SolveStatus::kInfeasible) {    // already checked with the rules of
    s.farkas_dual = p.farkas;                    // farkas_proves_infeasible
  } else if (s.status == SolveStatus::kUnbounded ||
             s.status == SolveStatus::kInfeasibleOrUnbounded) {
    s.primal_ray = p.ray;                        // ... and of ray_proves_unbounded
  }
  s.iterations = p.r.iterations;
  s.objective = p.r.objective;                   // original sense, offset included
  s.solve_seconds = p.r.total_seconds;
  s.dual_bound = p.r.dual_bound;
  s.message = p.r.message;
  if (measured_here) {
    s.recompute_quality(model);                  // measured, never assumed
  } else {
    const sankhya_pdhg_quality& q = p.r.quality;
    s.primal_infeasibility = q.primal_infeasibility;
    s.primal_infeasibility_scaled = q.primal_infeasibility_scaled;
    s.dual_infeasibility = q.dual_infeasibility;
    s.dual_infeasibility_scaled = q.dual_infeasibility_scaled;
    s.complementarity_violation = q.complementarity_violation;
    s.absolute_gap = q.absolute_gap;
    s.relative_gap = q.relative_gap;
  }
  return std::move(s);
}

}  // namespace

Solution solve_pdhg_gpu(const Model& model, const Options& options, Logger& logger) {
  Pending p;
  bind(p, model, "pdhg-gpu");
  const sankhya_pdhg_problem prob = problem_view(model);
  const sankhya_pdhg_params q = params_from(options);
  if (sankhya_pdhg_gpu_solve(&prob, &q, &p.r) != SANKHYA_GPU_SUCCESS)
    return failed(p, "GPU PDHG");
  logger.info("GPU PDHG: {} iterations, {} restarts, {:.3f} s on the device", p.r.iterations,
              p.r.restarts, p.r.solve_seconds);
  return finish(p, model, true);
}

// Many independent LPs (a scenario sweep, a decomposition's subproblems) in one call. The
// answers carry the quality block the device measured, so none is re-measured on the host.
std::vector<Solution> solve_pdhg_gpu_batch(const std::vector<const Model*>& models,
                                           const Options& options, Logger& logger) {
  std::vector<Pending> pending(models.size());
  std::vector<sankhya_pdhg_problem> probs;
  std::vector<sankhya_pdhg_result> results;
  for (std::size_t k = 0; k < models.size(); ++k) {
    bind(pending[k], *models[k], "pdhg-gpu");
    probs.push_back(problem_view(*models[k]));
    results.push_back(pending[k].r);
  }
  const sankhya_pdhg_params q = params_from(options);
  const int rc = sankhya_pdhg_gpu_batch_solve(probs.data(), static_cast<int32_t>(probs.size()),
                                              &q, results.data());
  std::vector<Solution> out;
  for (std::size_t k = 0; k < models.size(); ++k) {
    pending[k].r = results[k];
    out.push_back(rc == SANKHYA_GPU_SUCCESS ? finish(pending[k], *models[k], false)
                                            : failed(pending[k], "GPU PDHG"));
  }
  logger.info("GPU PDHG batch: {} LPs", models.size());
  return out;
}

// The convex-QP successor of qp::solve_convex_qp: the Hessian's lower triangle as the model
// stores it, qp_tolerance as the tolerance.
Solution solve_convex_qp_gpu(const Model& model, const Options& options, Logger& logger) {
  Pending p;
  bind(p, model, "qp-gpu");
  const sankhya_pdhg_problem prob = problem_view(model);
  sankhya_pdhg_params q = params_from(options);
  q.tolerance = options.get_double("qp_tolerance");
  const SparseMatrix& h = model.hessian;
  const sankhya_qp_hessian qh{h.num_nonzeros(), h.column_starts().data(),
                              h.row_indices().data(), h.values().data()};
  if (sankhya_qp_gpu_solve(&prob, &qh, &q, &p.r) != SANKHYA_GPU_SUCCESS)
    return failed(p, "GPU QP");
  logger.info("GPU QP: {} iterations, {:.3f} s on the device", p.r.iterations,
              p.r.solve_seconds);
  return finish(p, model, true);
}

}  // namespace sankhya::pdhg
