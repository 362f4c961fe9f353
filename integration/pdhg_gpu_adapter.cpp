// The reference-side adapter: the one translation unit a maintainer adds to the SANKHYA solver
// (as src/gpu/pdhg_gpu_adapter.cpp, compiled when the GPU backend is enabled) so that
// run_lp_engine (src/core/solve.cpp:385-395) can call the GPU engine where it calls
// pdhg::solve_pdhg (include/sankhya/pdhg.hpp:15). It turns the reference's Model and Options
// into the C-ABI structs of include/sankhya_pdhg_gpu.h and the result back into a Solution,
// using only the reference's own types and that header.
//
// Options: the six PDHG rows the reference already has are read as they are. The GPU rows
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

}  // namespace

Solution solve_pdhg_gpu(const Model& model, const Options& options, Logger& logger) {
  Solution s;
  s.allocate_for(model);
  s.algorithm = "pdhg-gpu";                      // verify.cpp:85-89 looks for "gpu"
  const SparseMatrix& a = model.matrix;          // frozen CSC, sparse.hpp:109-112
  sankhya_pdhg_problem p{model.num_rows(), model.num_cols(), model.num_nonzeros(),
                         a.column_starts().data(), a.row_indices().data(), a.values().data(),
                         model.col_cost.data(), model.col_lower.data(), model.col_upper.data(),
                         model.row_lower.data(), model.row_upper.data(),
                         model.sense == ObjSense::kMaximize, model.objective_offset};
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
  std::vector<double> farkas(model.num_rows()), ray(model.num_cols());
  sankhya_pdhg_result r{};
  r.col_value = s.col_value.data();
  r.row_dual = s.row_dual.data();
  r.col_dual = s.col_dual.data();
  r.farkas_dual = farkas.data();                 // filled when the status is INFEASIBLE
  r.primal_ray = ray.data();                     // filled when a ray is reported
  const int rc = sankhya_pdhg_gpu_solve(&p, &q, &r);
  if (rc != SANKHYA_GPU_SUCCESS) {               // no CPU fallback: the failure is the answer
    s.status = SolveStatus::kNumericalError;
    s.message = std::string("GPU PDHG: ") + sankhya_pdhg_gpu_last_error();
    return s;
  }
  s.status = to_solve_status(r.status);
  if (s.status == SolveStatus::kInfeasible) {    // already checked with the rules of
    s.farkas_dual = farkas;                      // farkas_proves_infeasible
  } else if (s.status == SolveStatus::kUnbounded ||
             s.status == SolveStatus::kInfeasibleOrUnbounded) {
    s.primal_ray = ray;                          // ... and of ray_proves_unbounded
  }
  s.iterations = r.iterations;
  s.primal_infeasibility = r.primal_infeasibility;  // the device's recompute_quality figure
  s.solve_seconds = r.total_seconds;
  s.dual_bound = r.dual_bound;
  s.message = r.message;
  s.recompute_quality(model);                    // pdhg.cpp:716: measured, never assumed
  logger.info("GPU PDHG: {} iterations, {} restarts, {:.3f} s on the device", r.iterations,
              r.restarts, r.solve_seconds);
  return s;
}

}  // namespace sankhya::pdhg
