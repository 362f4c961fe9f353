// Runs the reference-side adapter (integration/pdhg_gpu_adapter.cpp) as the reference solver
// would: a Model built with the reference's own API (the way tests/unit/test_pdhg.cpp builds
// its LPs), the reference's default Options, its Logger. Linked against the reference's
// objects and this library; prints one line for tests/test_integration_adapter.py:
//   status=<sankhya::to_string(status)> algorithm=<...> iterations=<...> objective=<...>
//   message=<...>
#include <cstdio>
#include <string>
#include <vector>

#include "sankhya/logging.hpp"
#include "sankhya/model.hpp"
#include "sankhya/options.hpp"

namespace sankhya::pdhg {
Solution solve_pdhg_gpu(const Model& model, const Options& options, Logger& logger);
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
  Logger logger(stdout, LogLevel::kWarning);
  const Solution s = pdhg::solve_pdhg_gpu(model, options, logger);
  std::printf("status=%s algorithm=%s iterations=%lld objective=%.17g message=%s\n",
              to_string(s.status), s.algorithm.c_str(), static_cast<long long>(s.iterations),
              s.objective, s.message.c_str());
  return 0;
}
