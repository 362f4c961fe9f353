// Host-side preparation of one LP for the PDHG kernels: validation, diagonal scaling,
// permuted CSR copies of A and A', and the SpMV work partition.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "sankhya_pdhg_gpu.h"

namespace sih26 {

// An error that ends a call: `code` is a sankhya_pdhg_gpu_status.
struct Failure {
  int code;
  std::string message;
};

bool host_finite_bound(double v);

// The reference's certificate checks (src/core/certificate.cpp:29-119 and :121-218) on the
// original problem: every certificate is re-checked with these before it is reported.
bool farkas_holds(const sankhya_pdhg_problem& p, const std::vector<double>& y);
bool ray_holds(const sankhya_pdhg_problem& p, const std::vector<double>& d);
// Cleans a primal-ray candidate taken from PDHG iterates (see pdhg_host.cpp); false when it
// cannot. The result still has to pass ray_holds.
bool repair_ray(const sankhya_pdhg_problem& p, std::vector<double>& d);

// Structural checks of the C-ABI input (sizes, pointers, CSC well-formedness). Throws Failure
// with SANKHYA_GPU_INVALID_ARGUMENT; these are inputs the reference's frozen SparseMatrix can
// never hold.
void check_structure(const sankhya_pdhg_problem& p);

// Model::validate for an LP (src/core/model.cpp:125-210): returns "" or the first problem.
// Runs after check_structure has passed (it reads each column's range of the arrays).
std::string validate_model(const sankhya_pdhg_problem& p);

// build_scaling (src/la/scaling.cpp:111-158): 10 Ruiz rounds then one Pock-Chambolle round,
// in the reference's order of operations, so Dr and Dc are bit-identical to it.
struct Scaling {
  std::vector<double> dr, dc, values, cost, cl, cu, rl, ru;
};
Scaling build_scaling(const sankhya_pdhg_problem& p, const std::vector<double>& min_cost,
                      int ruiz_rounds);

// Rows of A and of A' each sorted by nonzero count, longest first (stable), with CSR copies
// in that order whose column indices point into the other permuted space.
struct PermutedLp {
  int m = 0, n = 0;
  long long nnz = 0;
  std::vector<int> row_perm, col_perm;  // position -> original index
  std::vector<int> a_ptr, a_idx, at_ptr, at_idx;
  std::vector<double> a_val, at_val;
};
PermutedLp permute(const sankhya_pdhg_problem& p, const std::vector<double>& scaled_values);

// Work partition of one CSR matrix over G blocks (see Part in pdhg_kernels.cuh). The schedule
// knobs: rows of at most stream_row_max nonzeros go to stream items (a warp loads a whole item
// at once, lane r sums row r); longer rows up to 512 nonzeros get a power-of-two lane group
// with at most nnz_per_lane nonzeros per lane.
struct Schedule {
  int stream_row_max = 32;
  int nnz_per_lane = 16;
};
// The result's quality block from the device's quality slots (kQualitySlots in
// pdhg_kernels.cuh), the objective and the dual bound: the row-price terms take the dual-norm
// scale max(1, max |row_dual|) here, and the gaps follow src/core/model.cpp:419-421.
sankhya_pdhg_quality quality_from_slots(const double* slots, double objective, double dual_bound);

struct HostPart {
  std::vector<int> blk_seg_begin, blk_long_begin, blk_item_begin;
  std::vector<int4> segs, longs, items;
  long long sell_entries = 0;  // sliced partitions: entries of the slice arrays
};
// sliced = true: the rows that would go to stream items go to slices instead ({row_begin,
// row_end, -L, offset}: up to 32 consecutive rows stored column-major in separate arrays,
// entry k of row row_begin + l at offset + k * rows + l, L the longest row), which one thread
// per row sums with coalesced loads and no shared memory (the iteration kernel's layout).
HostPart partition(const std::vector<int>& ptr, int G, int warps_per_block, int lanes_override,
                   Schedule sched = Schedule{}, bool sliced = false);

// The autotuner's cache (one line per key, see pdhg_host.cpp). The key is built from the
// row-length statistics of A and A' (mean, max, coefficient of variation, share of nonzeros
// in 33-512 and >512 nonzero rows), power-of-two size buckets, the grid and the value width.
std::string autotune_key(const PermutedLp& q, int G, int sms, int value_bytes);
std::string autotune_cache_path();
bool autotune_lookup(const std::string& path, const std::string& key, Schedule* a, Schedule* at);
// The served engine's chunk length for an LP family (one line per key: key, chunk, the LPs
// per second it measured; the last line of a key wins).
bool chunk_lookup(const std::string& path, const std::string& key, long long* chunk);
void chunk_store(const std::string& path, const std::string& key, long long chunk, double rate);
// Key of a family of served LPs: the SM count, the launch slots, and the median nonzeros and
// median nonzeros per row of a sample of its LPs (power-of-two and two-digit buckets).
std::string chunk_key(int sms, int slots, std::vector<long long> nnz, std::vector<double> per_row);
void autotune_store(const std::string& path, const std::string& key, const Schedule& a,
                    const Schedule& at, double us_a, double us_at);

// mt19937 + uniform_real_distribution<double>(lo, hi) as libstdc++ draws it: the random start
// of estimate_spectral_norm (src/la/scaling.cpp:168-171).
void uniform_draws(uint32_t seed, double lo, double hi, size_t count, double* out);

}  // namespace sih26
