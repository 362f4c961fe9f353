// Runs the reference-side adapter (integration/pdhg_gpu_adapter.cpp) as the reference solver
// would: Models built with the reference's own API (the way tests/unit/test_pdhg.cpp builds
// its LPs), the reference's default Options, its Logger. Linked against the reference's
// objects and this library; prints one line per adapter call for
// tests/test_integration_adapter.py:
//   call=<lp|batch0|batch1|qp> status=<sankhya::to_string(status)> algorithm=<...>
//   iterations=<...> objective=<...> message=<...>
#include <cstdio>
#include <string>
#include <vector>

#include "sankhya/logging.hpp"
#include "sankhya/model.hpp"
#include "sankhya/options.hpp"

namespace sankhya::pdhg {
Solution solve_pdhg_gpu(const Model& model, const Options& options, Logger& logger);
std::vector<Solution> solve_pdhg_gpu_batch(const std::vector<const Model*>& models,
                                           const Options& options, Logger& logger);
Solution solve_convex_qp_gpu(const Model& model, const Options& options, Logger& logger);
}

static void report(const char* call, const sankhya::Solution& s) {
  std::printf("call=%s status=%s algorithm=%s iterations=%lld objective=%.17g message=%s\n",
              call, sankhya::to_string(s.status), s.algorithm.c_str(),
              static_cast<long long>(s.iterations), s.objective, s.message.c_str());
}

int main() {
  using namespace sankhya;
  // min -3x - 5y  s.t.  x <= 4, 2y <= 12, 3x + 2y <= 18, x, y >= 0: optimum -36 at (2, 6)
  const std::vector<std::vector<double>> rows = {{1.0, 0.0}, {0.0, 2.0}, {3.0, 2.0}};
  Model model;
  model.col_cost = {-3.0, -5.0};
  model.col_lower = {0.0, 0.0};
  model.col_upper = {kInfinity, kInfinity};
  model.col_type.assign(2, VarType::kContinuous);
  model.row_lower = {-kInfinity, -kInfinity, -kInfinity};
  model.row_upper = {4.0, 12.0, 18.0};
  model.matrix.reset(3, 2);
  for (Index i = 0; i < 3; ++i)
    for (Index j = 0; j < 2; ++j)
      if (rows[i][j] != 0.0) model.matrix.add_entry(i, j, rows[i][j]);
  model.matrix.finalize();
  model.hessian.reset(2, 2);
  model.hessian.finalize();
  if (!model.validate().empty()) {
    std::printf("status=bad_model message=%s\n", model.validate().c_str());
    return 1;
  }
  Options options;
  options.set_bool("log_to_console", false);
  options.set_double("pdhg_tolerance", 1e-8);
  options.set_double("qp_tolerance", 1e-8);
  Logger logger(stdout, LogLevel::kWarning);
  report("lp", pdhg::solve_pdhg_gpu(model, options, logger));
  const std::vector<Solution> batch = pdhg::solve_pdhg_gpu_batch({&model, &model}, options,
                                                                  logger);
  report("batch0", batch.at(0));
  report("batch1", batch.at(1));
  // the same rows with 1/2 (x^2 + y^2) added: (3, 5) projected onto 3x + 2y <= 18, optimum
  // (36/13, 63/13) at 1/26 - 17
  Model qp = model;
  qp.hessian.reset(2, 2);
  qp.hessian.add_entry(0, 0, 1.0);
  qp.hessian.add_entry(1, 1, 1.0);
  qp.hessian.finalize();
  report("qp", pdhg::solve_convex_qp_gpu(qp, options, logger));
  return 0;
}
