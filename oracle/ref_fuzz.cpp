// TEST INFRASTRUCTURE ONLY -- never linked into the product.
//
// The reference's cross-engine gate draws its instances from its own test generator:
// tests/unit/test_pdhg.cpp:178-222 runs 120 instances of oracle::kkt_lp
// (tests/oracles/lp_generator.cpp:122-189) from std::mt19937_64(20260904) with at most 6 rows
// and 6 columns, converted by oracle::to_model (tests/oracles/rational_simplex.hpp:59). This
// entry point replays that sequence with the reference's own generator sources (compiled in
// place by oracle/Makefile, target `ref`) and hands instance `index` back in the reference's
// CSC convention, with its analytic optimum, so the fixture made from it holds exactly the
// instances the reference's gate solves.
#include <cstdint>
#include <cstring>
#include <random>

#include "oracles/lp_generator.hpp"
#include "oracles/rational_simplex.hpp"
#include "sankhya/model.hpp"

extern "C" {

struct ref_fuzz_lp {
  std::int32_t num_rows;
  std::int32_t num_cols;
  std::int32_t num_nonzeros;
  std::int32_t* col_starts;
  std::int32_t* row_indices;
  double* values;
  double* cost;
  double* col_lower;
  double* col_upper;
  double* row_lower;
  double* row_upper;
  std::int32_t maximize;
  double objective_offset;
};

/// Instance `index` (0-based) of the kkt_lp sequence from mt19937_64(seed) with the given row
/// and column caps. Call once with col_starts NULL for the sizes, then with arrays of those
/// sizes. *optimal receives the instance's analytic optimal objective.
int ref_kkt_instance(std::uint64_t seed, int max_rows, int max_cols, int index, ref_fuzz_lp* lp,
                     double* optimal) {
  using namespace sankhya;
  try {
    std::mt19937_64 rng(seed);
    oracle::GeneratorConfig config;
    config.max_rows = max_rows;
    config.max_cols = max_cols;
    oracle::KktInstance instance;
    for (int k = 0; k <= index; ++k) instance = oracle::kkt_lp(rng, config);
    const Model model = oracle::to_model(instance.lp);
    *optimal = static_cast<double>(instance.optimal_objective);
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
    std::memcpy(lp->col_starts, model.matrix.column_starts().data(), (n + 1) * 4);
    std::memcpy(lp->row_indices, model.matrix.row_indices().data(),
                model.matrix.row_indices().size() * 4);
    std::memcpy(lp->values, model.matrix.values().data(), model.matrix.values().size() * 8);
    std::memcpy(lp->cost, model.col_cost.data(), n * 8);
    std::memcpy(lp->col_lower, model.col_lower.data(), n * 8);
    std::memcpy(lp->col_upper, model.col_upper.data(), n * 8);
    std::memcpy(lp->row_lower, model.row_lower.data(), m * 8);
    std::memcpy(lp->row_upper, model.row_upper.data(), m * 8);
    return 0;
  } catch (...) {
    return 1;
  }
}

}  // extern "C"
