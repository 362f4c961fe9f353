// Convex QP on the GPU behind sankhya_qp_gpu_solve (include/sankhya_pdhg_gpu.h): the reference's
// Condat-Vu method (src/qp/qp_condat_vu.cpp:150-323) on the LP engine's fused SpMV phases.
//
//   x'   = proj_box(x - tau (c_s + Q_s x + A'y))        c_s = sense c, Q_s = sense Q
//   xbar = 2 x' - x
//   y'   = v - sigma proj_C(v / sigma),  v = y + sigma A xbar
//
// Phase P runs over the rows of C = [A' | Q_s] (one row per column of the LP), gathering y for
// the A' part and x for the Q part, so the gradient is one fused row sum; phase D runs over the
// rows of A gathering xbar. Every 50 iterations (the reference's cadence, counted the same way)
// two more passes measure the termination residuals: max_i |Ax - proj(Ax)| and
// max_j |x - proj(x - gradient)|. Steps come from the reference's own power iterations for
// ||A|| and ||Q||, restated on the host in its order of operations, so tau and sigma are the
// reference's to the bit. Everything is FP64, as in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pdhg_host.cuh"
#include "pdhg_kernels.cuh"
#include "sankhya_pdhg_gpu.h"

namespace sih26 {

extern thread_local std::string g_last_error;

namespace {

#define SIH26_QCUDA(expr, code)                                                          \
  do {                                                                                   \
    const cudaError_t e_ = (expr);                                                       \
    if (e_ != cudaSuccess)                                                               \
      throw Failure{code, std::string(#expr) + ": " + cudaGetErrorString(e_)};           \
  } while (0)

// ---- device -----------------------------------------------------------------------------

struct QpDev {
  int m, n;
  Csr<double> A, C;  // A in permuted rows; C = [A' | Q_s] in permuted columns
  Part pa, pc;
  const double* c;   // sense c, permuted
  const double* cl;
  const double* cu;
  const double* rl;
  const double* ru;
  double* x[2];
  double* xbar;
  double* y[2];
  double* partials;  // [G][kPartSlots]
  Ctrl* ctrl;        // iteration, state, the two residuals in best.absolute_primal / _dual
  GridBarrier bar;
  double tau, sigma, tolerance;
  long long iteration_limit;
};

// sum_k C_jk z_k with z = [y; x]
struct CombinedGather {
  const double* y;
  const double* x;
  int m;
  __device__ __forceinline__ double at(int k) const { return k < m ? ld(y + k) : ld(x + (k - m)); }
  __device__ __forceinline__ void add(double (&s)[1], double a, int k) const { s[0] += a * at(k); }
  __device__ __forceinline__ double product(int, double a, int k) const { return a * at(k); }
};

struct QpPrimal {
  const double* x;
  double* xn;
  double* xbar;
  const double* c;
  const double* cl;
  const double* cu;
  double tau;
  struct In {
    double xo, c, lo, hi;
  };
  __device__ __forceinline__ In load(int j) const {
    return In{ld(x + j), __ldg(c + j), __ldg(cl + j), __ldg(cu + j)};
  }
  __device__ __forceinline__ void apply(int j, const double (&s)[1], const In& v, double (&)[1]) const {
    const double xp = project(v.xo - tau * (v.c + s[0]), v.lo, v.hi);
    xn[j] = xp;
    xbar[j] = 2.0 * xp - v.xo;
  }
};

struct QpDual {
  const double* y;
  double* yn;
  const double* rl;
  const double* ru;
  double sigma;
  struct In {
    double yo, lo, hi;
  };
  __device__ __forceinline__ In load(int i) const { return In{ld(y + i), __ldg(rl + i), __ldg(ru + i)}; }
  __device__ __forceinline__ void apply(int i, const double (&s)[1], const In& v, double (&)[1]) const {
    const double u = v.yo + sigma * s[0];
    yn[i] = u - sigma * project(u / sigma, v.lo, v.hi);
  }
};

// termination measures (qp_condat_vu.cpp:263-289)
struct QpPrimalResidual {
  const double* rl;
  const double* ru;
  struct In {
    double lo, hi;
  };
  __device__ __forceinline__ In load(int i) const { return In{__ldg(rl + i), __ldg(ru + i)}; }
  __device__ __forceinline__ void apply(int, const double (&s)[1], const In& v, double (&acc)[2]) const {
    acc[0] = dmax(acc[0], fabs(s[0] - project(s[0], v.lo, v.hi)));
  }
};
struct QpDualResidual {
  const double* x;
  const double* c;
  const double* cl;
  const double* cu;
  struct In {
    double xo, c, lo, hi;
  };
  __device__ __forceinline__ In load(int j) const {
    return In{ld(x + j), __ldg(c + j), __ldg(cl + j), __ldg(cu + j)};
  }
  __device__ __forceinline__ void apply(int, const double (&s)[1], const In& v, double (&acc)[2]) const {
    const double g = v.c + s[0];
    acc[1] = dmax(acc[1], fabs(v.xo - project(v.xo - g, v.lo, v.hi)));
  }
};

// Cooperative: runs iterations until the limit, the chunk end or convergence. Ctrl fields
// used: iteration (the reference's loop counter), state, cur, best.absolute_primal/_dual.
__global__ void __launch_bounds__(kThreads, 2) qp_kernel(QpDev Q, long long max_steps) {
  __shared__ Ctrl c;
  __shared__ double sh[kWarps * 2];
  double* stream = warp_stream();
  if (threadIdx.x == 0) {
    c = *Q.ctrl;
    // read once per launch, before the first barrier, so every block sees the same flag
    c.time_up |= *((volatile int*)Q.bar.time_up);
  }
  __syncthreads();
  if (c.state != kRunning) return;
  const int G = gridDim.x;
  for (long long step = 0; step < max_steps; ++step) {
    if (c.iteration >= Q.iteration_limit) {
      if (threadIdx.x == 0) c.state = kIterationLimit;
      break;
    }
    if (c.time_up) {
      if (threadIdx.x == 0) c.state = kTimeLimit;
      break;
    }
    const int cur = c.cur, nxt = cur ^ 1;
    double dummy[1] = {0.0};
    run_phase<1, 1>(Q.C.ptr, Q.C.idx, Q.C.val, Q.pc, CombinedGather{Q.y[cur], Q.x[cur], Q.m},
                    QpPrimal{Q.x[cur], Q.x[nxt], Q.xbar, Q.c, Q.cl, Q.cu, Q.tau}, dummy, stream);
    if (!grid_barrier(Q.bar)) goto device_error;
    run_phase<1, 1>(Q.A.ptr, Q.A.idx, Q.A.val, Q.pa, Gather1<double>{Q.xbar},
                    QpDual{Q.y[cur], Q.y[nxt], Q.rl, Q.ru, Q.sigma}, dummy, stream);
    if (!grid_barrier(Q.bar)) goto device_error;
    // the reference checks after the step when its counter is a multiple of 50, then counts
    if (c.iteration % 50 == 0) {
      double acc[2] = {0.0, 0.0};
      run_phase<1, 2>(Q.A.ptr, Q.A.idx, Q.A.val, Q.pa, Gather1<double>{Q.x[nxt]},
                      QpPrimalResidual{Q.rl, Q.ru}, acc, stream);
      run_phase<1, 2>(Q.C.ptr, Q.C.idx, Q.C.val, Q.pc, CombinedGather{Q.y[nxt], Q.x[nxt], Q.m},
                      QpDualResidual{Q.x[nxt], Q.c, Q.cl, Q.cu}, acc, stream);
      block_reduce<2, 3u>(acc, sh);
      write_partials(Q.partials, 0, acc, 2);
      if (!grid_barrier(Q.bar)) goto device_error;
      double tot[2];
      reduce_partials<2, 3u>(Q.partials, 0, tot, sh);
      if (threadIdx.x == 0) {
        c.best.absolute_primal = tot[0];
        c.best.absolute_dual = tot[1];
        if (tot[0] <= Q.tolerance && tot[1] <= Q.tolerance) {
          c.state = kConverged;
          c.converged = 1;
        }
      }
    }
    if (threadIdx.x == 0) {
      c.cur = nxt;
      if (c.state != kConverged) ++c.iteration;
    }
    __syncthreads();
    if (c.state != kRunning) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *Q.ctrl = c;
  return;
device_error:
  if (blockIdx.x == 0 && threadIdx.x == 0) Q.ctrl->state = kDeviceError;
}

// ---- host --------------------------------------------------------------------------------

// The reference's spectral_norm (qp_condat_vu.cpp:64-97): 20 power iterations on A'A from
// mt19937(26119) uniform(-1, 1), multiply_add / transpose_multiply_add in their order.
double qp_norm_a(const sankhya_pdhg_problem& p) {
  const int m = p.num_rows, n = p.num_cols;
  if (m == 0 || n == 0 || p.num_nonzeros == 0) return 0.0;
  std::vector<double> v(n), av(m);
  uniform_draws(26119u, -1.0, 1.0, n, v.data());
  double estimate = 0.0;
  for (int it = 0; it < 20; ++it) {
    double norm = 0.0;
    for (double t : v) norm += t * t;
    norm = std::sqrt(norm);
    if (norm <= 0.0) return 0.0;
    for (double& t : v) t /= norm;
    std::fill(av.begin(), av.end(), 0.0);
    for (int j = 0; j < n; ++j) {
      const double xj = 1.0 * v[j];
      if (xj == 0.0) continue;
      for (int k = p.col_starts[j]; k < p.col_starts[j + 1]; ++k) av[p.row_indices[k]] += p.values[k] * xj;
    }
    std::fill(v.begin(), v.end(), 0.0);
    for (int j = 0; j < n; ++j) {
      double dot = 0.0;
      for (int k = p.col_starts[j]; k < p.col_starts[j + 1]; ++k) dot += p.values[k] * av[p.row_indices[k]];
      v[j] += 1.0 * dot;
    }
    double next = 0.0;
    for (double t : v) next += t * t;
    estimate = std::sqrt(std::sqrt(next));
  }
  return estimate;
}

// Q v from the stored lower triangle (qp_condat_vu.cpp:137-150)
void qp_hessian_multiply(int n, const sankhya_qp_hessian& h, const std::vector<double>& v,
                         std::vector<double>& out) {
  std::fill(out.begin(), out.end(), 0.0);
  for (int j = 0; j < n; ++j) {
    for (int k = h.col_starts[j]; k < h.col_starts[j + 1]; ++k) {
      const int i = h.row_indices[k];
      const double value = h.values[k];
      out[i] += value * v[j];
      if (i != j) out[j] += value * v[i];
    }
  }
}

// The reference's hessian_norm (qp_condat_vu.cpp:101-134): 20 power iterations on Q from
// mt19937(20260826) uniform(-1, 1); the estimate is |v'Qv| with v normalised.
double qp_norm_q(int n, const sankhya_qp_hessian& h) {
  if (h.num_nonzeros == 0 || n == 0) return 0.0;
  std::vector<double> v(n), qv(n);
  uniform_draws(20260826u, -1.0, 1.0, n, v.data());
  double estimate = 0.0;
  for (int it = 0; it < 20; ++it) {
    double norm = 0.0;
    for (double t : v) norm += t * t;
    norm = std::sqrt(norm);
    if (norm <= 0.0) return 0.0;
    for (double& t : v) t /= norm;
    qp_hessian_multiply(n, h, v, qv);
    double next = 0.0;
    for (int i = 0; i < n; ++i) next += qv[i] * v[i];
    estimate = std::fabs(next);
    v = qv;
  }
  return estimate;
}

// check_convexity (src/qp/convexity.cpp:30-134): dense LDL' of sense * Q without interchanges,
// up to 2,000 columns. Returns "" when convex, else the reason (the reference's wording).
std::string qp_convexity(int n, const sankhya_qp_hessian& h, double sense) {
  if (h.num_nonzeros == 0) return "";
  constexpr int kDenseLimit = 2000;
  constexpr double kPivotSlackFactor = 1e-10;
  char buf[256];
  if (n > kDenseLimit) {
    std::snprintf(buf, sizeof buf,
                  "convexity could not be established: %d columns exceeds the %d the dense "
                  "convexity test can decide",
                  n, kDenseLimit);
    return buf;
  }
  const size_t un = static_cast<size_t>(n);
  std::vector<double> q(un * un, 0.0);
  double largest_diagonal = 0.0;
  for (int j = 0; j < n; ++j) {
    for (int k = h.col_starts[j]; k < h.col_starts[j + 1]; ++k) {
      const int i = h.row_indices[k];
      const double value = sense * h.values[k];
      q[static_cast<size_t>(i) * un + j] = value;
      q[static_cast<size_t>(j) * un + i] = value;
      if (i == j) largest_diagonal = std::max(largest_diagonal, std::fabs(value));
    }
  }
  for (int i = 0; i < n; ++i) {
    const double d = q[static_cast<size_t>(i) * un + i];
    if (d < -kPivotSlackFactor * std::max(1.0, largest_diagonal)) {
      std::snprintf(buf, sizeof buf,
                    "the quadratic objective is not convex: the Hessian diagonal for column %d "
                    "is %.6g in minimization sense",
                    i, d);
      return buf;
    }
  }
  const double slack = kPivotSlackFactor * std::max(1.0, largest_diagonal);
  std::vector<double> l(un * un, 0.0), d(un, 0.0);
  for (int j = 0; j < n; ++j) {
    double pivot = q[static_cast<size_t>(j) * un + j];
    for (int k = 0; k < j; ++k) pivot -= l[j * un + k] * l[j * un + k] * d[k];
    if (pivot < -slack) {
      std::snprintf(buf, sizeof buf,
                    "the quadratic objective is not convex: LDL^T reached a pivot of %.6g at "
                    "column %d",
                    pivot, j);
      return buf;
    }
    if (pivot <= slack) {
      d[j] = 0.0;
      for (int i = j + 1; i < n; ++i) l[i * un + j] = 0.0;
      continue;
    }
    d[j] = pivot;
    // the rows below the pivot are independent: each keeps the reference's order over k
#pragma omp parallel for schedule(static) if (n - j > 256)
    for (int i = j + 1; i < n; ++i) {
      double sum = q[i * un + j];
      for (int k = 0; k < j; ++k) sum -= l[i * un + k] * l[j * un + k] * d[k];
      l[i * un + j] = sum / pivot;
    }
  }
  return "";
}

void check_hessian(const sankhya_pdhg_problem& p, const sankhya_qp_hessian& h) {
  const auto bad = [](const std::string& why) { throw Failure{SANKHYA_GPU_INVALID_ARGUMENT, why}; };
  const int n = p.num_cols;
  if (h.num_nonzeros < 0) bad("negative Hessian size");
  if (!h.col_starts) bad("Hessian col_starts is NULL");
  if (h.num_nonzeros > 0 && (!h.row_indices || !h.values)) bad("Hessian arrays are NULL");
  if (h.col_starts[0] != 0 || h.col_starts[n] != h.num_nonzeros) bad("Hessian col_starts inconsistent");
  for (int j = 0; j < n; ++j) {
    if (h.col_starts[j + 1] < h.col_starts[j]) bad("Hessian col_starts decreases");
    for (int k = h.col_starts[j]; k < h.col_starts[j + 1]; ++k) {
      const int i = h.row_indices[k];
      if (i < j || i >= n) bad("the Hessian must be a lower triangle (row >= column < n)");
      if (k > h.col_starts[j] && i <= h.row_indices[k - 1]) bad("Hessian rows not ascending");
      if (!std::isfinite(h.values[k])) bad("non-finite Hessian entry");
    }
  }
}

template <class T>
T* dev_upload(std::vector<void*>& owned, const std::vector<T>& h) {
  void* p = nullptr;
  SIH26_QCUDA(cudaMalloc(&p, std::max<size_t>(1, h.size()) * sizeof(T)), SANKHYA_GPU_OUT_OF_MEMORY);
  owned.push_back(p);
  if (!h.empty())
    SIH26_QCUDA(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), SANKHYA_GPU_COPY_FAILED);
  return static_cast<T*>(p);
}

Part dev_part(std::vector<void*>& owned, const HostPart& hp) {
  Part p;
  p.blk_seg_begin = dev_upload(owned, hp.blk_seg_begin);
  p.segs = dev_upload(owned, hp.segs);
  p.blk_long_begin = dev_upload(owned, hp.blk_long_begin);
  p.longs = dev_upload(owned, hp.longs);
  p.blk_item_begin = dev_upload(owned, hp.blk_item_begin);
  p.items = dev_upload(owned, hp.items);
  p.seg_sum = dev_upload(owned, std::vector<double>(hp.segs.size() * 2 + 1, 0.0));
  return p;
}

std::vector<int> order_desc(const std::vector<int>& len) {
  std::vector<int> order(len.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = static_cast<int>(i);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return len[a] > len[b]; });
  return order;
}

int qp_solve_impl(const sankhya_pdhg_problem& prob, const sankhya_qp_hessian& hes,
                  const sankhya_pdhg_params& prm, sankhya_pdhg_result* res) {
  using Clock = std::chrono::steady_clock;
  const Clock::time_point t0 = Clock::now();
  const auto since = [&]() { return std::chrono::duration<double>(Clock::now() - t0).count(); };
  check_structure(prob);
  check_hessian(prob, hes);
  const int m = prob.num_rows, n = prob.num_cols;
  res->status = SANKHYA_PDHG_NOT_SOLVED;
  res->converged = 0;
  res->iterations = res->attempts = res->restarts = res->evaluations = res->fp32_iterations = 0;
  res->message[0] = '\0';
  const std::string why = validate_model(prob);
  const double sense = prob.maximize ? -1.0 : 1.0;
  std::string convex = prm.qp_assume_convex ? std::string() : qp_convexity(n, hes, sense);
  if (!why.empty() || !convex.empty()) {
    res->status = SANKHYA_PDHG_MODEL_ERROR;
    std::snprintf(res->message, sizeof res->message, "%s", (why.empty() ? convex : why).c_str());
    return SANKHYA_GPU_SUCCESS;
  }
  int devices = 0;
  if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0)
    throw Failure{SANKHYA_GPU_NO_COMPATIBLE_DEVICE, "no CUDA device is visible"};
  if (prm.device < 0 || prm.device >= devices)
    throw Failure{SANKHYA_GPU_INVALID_ARGUMENT, "device ordinal out of range"};
  SIH26_QCUDA(cudaSetDevice(prm.device), SANKHYA_GPU_INIT_FAILED);
  cudaDeviceProp props{};
  SIH26_QCUDA(cudaGetDeviceProperties(&props, prm.device), SANKHYA_GPU_INIT_FAILED);
  if (props.major < 10)
    throw Failure{SANKHYA_GPU_NO_COMPATIBLE_DEVICE, "this library is built for sm_100a (B200)"};

  // ---- step sizes, as the reference (qp_condat_vu.cpp:183-196) ----
  const double norm_a = qp_norm_a(prob);
  const double norm_q = qp_norm_q(n, hes);
  const double margin = 1.05;
  const double lq = margin * norm_q;
  const double a2 = margin * margin * std::max(norm_a * norm_a, 1e-12);
  const double tau = 1.0 / (lq / 2.0 + std::sqrt(a2) + 1e-12);
  const double sigma = (m > 0) ? (1.0 / tau - lq / 2.0) / (2.0 * a2) : 0.0;
  const double tolerance = prm.tolerance > 0.0 ? prm.tolerance : 1e-8;

  // ---- layout: rows of A by length; columns by the length of their row of C = [A' | Q_s] ----
  std::vector<int> rlen(m, 0), clen(n, 0);
  std::vector<std::vector<std::pair<int, double>>> qrow(n);  // full symmetric Q_s, by row
  for (int j = 0; j < n; ++j) {
    clen[j] += prob.col_starts[j + 1] - prob.col_starts[j];
    for (int k = prob.col_starts[j]; k < prob.col_starts[j + 1]; ++k) ++rlen[prob.row_indices[k]];
    for (int k = hes.col_starts[j]; k < hes.col_starts[j + 1]; ++k) {
      const int i = hes.row_indices[k];
      const double v = sense * hes.values[k];
      qrow[i].push_back({j, v});
      if (i != j) qrow[j].push_back({i, v});
    }
  }
  for (int j = 0; j < n; ++j) clen[j] += static_cast<int>(qrow[j].size());
  const std::vector<int> row_perm = order_desc(rlen), col_perm = order_desc(clen);
  std::vector<int> row_pos(m), col_pos(n);
  for (int t = 0; t < m; ++t) row_pos[row_perm[t]] = t;
  for (int t = 0; t < n; ++t) col_pos[col_perm[t]] = t;
  // A in permuted rows, entries in ascending permuted column
  std::vector<int> a_ptr(m + 1, 0);
  for (int t = 0; t < m; ++t) a_ptr[t + 1] = a_ptr[t] + rlen[row_perm[t]];
  std::vector<int> a_idx(prob.num_nonzeros);
  std::vector<double> a_val(prob.num_nonzeros);
  {
    std::vector<int> next(a_ptr.begin(), a_ptr.end() - 1);
    for (int t = 0; t < n; ++t) {
      const int j = col_perm[t];
      for (int k = prob.col_starts[j]; k < prob.col_starts[j + 1]; ++k) {
        const int slot = next[row_pos[prob.row_indices[k]]]++;
        a_idx[slot] = t;
        a_val[slot] = prob.values[k];
      }
    }
  }
  // C in permuted columns: A' entries (permuted row positions, ascending), then Q_s entries
  // (m + permuted column positions, ascending)
  std::vector<int> c_ptr(n + 1, 0);
  for (int t = 0; t < n; ++t) c_ptr[t + 1] = c_ptr[t] + clen[col_perm[t]];
  std::vector<int> c_idx(c_ptr[n]);
  std::vector<double> c_val(c_ptr[n]);
  for (int t = 0; t < n; ++t) {
    const int j = col_perm[t];
    std::vector<std::pair<int, double>> a_part, q_part;
    for (int k = prob.col_starts[j]; k < prob.col_starts[j + 1]; ++k)
      a_part.push_back({row_pos[prob.row_indices[k]], prob.values[k]});
    for (const auto& e : qrow[j]) q_part.push_back({m + col_pos[e.first], e.second});
    std::sort(a_part.begin(), a_part.end());
    std::sort(q_part.begin(), q_part.end());
    int at = c_ptr[t];
    for (const auto& e : a_part) { c_idx[at] = e.first; c_val[at++] = e.second; }
    for (const auto& e : q_part) { c_idx[at] = e.first; c_val[at++] = e.second; }
  }
  std::vector<double> cs(n), cl(n), cu(n), rl(m), ru(m);
  for (int t = 0; t < n; ++t) {
    const int j = col_perm[t];
    cs[t] = sense * prob.cost[j];
    cl[t] = prob.col_lower[j];
    cu[t] = prob.col_upper[j];
  }
  for (int t = 0; t < m; ++t) {
    rl[t] = prob.row_lower[row_perm[t]];
    ru[t] = prob.row_upper[row_perm[t]];
  }
  std::vector<double> x0(n);
  for (int t = 0; t < n; ++t) {
    double v = 0.0;
    if (host_finite_bound(cl[t]) && v < cl[t]) v = cl[t];
    else if (host_finite_bound(cu[t]) && v > cu[t]) v = cu[t];
    x0[t] = v;
  }

  // ---- device ----
  int bpsm = 0;
  SIH26_QCUDA(cudaFuncSetAttribute(qp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)stream_smem_bytes()), SANKHYA_GPU_INIT_FAILED);
  SIH26_QCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, qp_kernel, kThreads, stream_smem_bytes()),
              SANKHYA_GPU_INIT_FAILED);
  if (bpsm < 1) throw Failure{SANKHYA_GPU_INIT_FAILED, "kernel does not fit on an SM"};
  int G = props.multiProcessorCount * std::min(bpsm, 2);
  const long long work = static_cast<long long>(c_ptr[n]) + prob.num_nonzeros + m + n;
  G = static_cast<int>(std::max<long long>(1, std::min<long long>(G, (work + 4095) / 4096)));

  std::vector<void*> owned;
  struct Owned {
    std::vector<void*>& v;
    ~Owned() { for (void* p : v) cudaFree(p); }
  } guard{owned};
  QpDev Q{};
  Q.m = m;
  Q.n = n;
  Q.A.ptr = dev_upload(owned, a_ptr);
  Q.A.idx = dev_upload(owned, a_idx);
  Q.A.val = Q.A.val64 = dev_upload(owned, a_val);
  Q.C.ptr = dev_upload(owned, c_ptr);
  Q.C.idx = dev_upload(owned, c_idx);
  Q.C.val = Q.C.val64 = dev_upload(owned, c_val);
  Q.pa = dev_part(owned, partition(a_ptr, G, kWarps, 0));
  Q.pc = dev_part(owned, partition(c_ptr, G, kWarps, 0));
  Q.c = dev_upload(owned, cs);
  Q.cl = dev_upload(owned, cl);
  Q.cu = dev_upload(owned, cu);
  Q.rl = dev_upload(owned, rl);
  Q.ru = dev_upload(owned, ru);
  Q.x[0] = dev_upload(owned, x0);
  Q.x[1] = dev_upload(owned, x0);
  Q.xbar = dev_upload(owned, std::vector<double>(n, 0.0));
  Q.y[0] = dev_upload(owned, std::vector<double>(m, 0.0));
  Q.y[1] = dev_upload(owned, std::vector<double>(m, 0.0));
  Q.partials = dev_upload(owned, std::vector<double>(static_cast<size_t>(G) * kPartSlots, 0.0));
  Ctrl c0{};
  c0.state = kRunning;
  c0.iteration_limit = prm.iteration_limit < 0 ? 1000000ll : prm.iteration_limit;
  Q.ctrl = dev_upload(owned, std::vector<Ctrl>(1, c0));
  std::vector<unsigned> bw(2, 0u);
  std::vector<int> fl(2, 0);
  unsigned* bar_words = dev_upload(owned, bw);
  int* flags = dev_upload(owned, fl);
  Q.bar = GridBarrier{bar_words, flags, 4000000000ull, flags + 1, 0ull, -1};
  Q.tau = tau;
  Q.sigma = sigma;
  Q.tolerance = tolerance;
  Q.iteration_limit = c0.iteration_limit;
  const bool timed = std::isfinite(prm.time_limit) && prm.time_limit > 0.0;

  cudaStream_t stream;
  SIH26_QCUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), SANKHYA_GPU_INIT_FAILED);
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{stream};
  Ctrl host{};
  long long steps = 256;
  long long launches = 0;
  for (;;) {
    void* args[] = {&Q, &steps};
    SIH26_QCUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(qp_kernel), dim3(G),
                                            dim3(kThreads), args, stream_smem_bytes(), stream),
                SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
    ++launches;
    SIH26_QCUDA(cudaMemcpyAsync(&host, Q.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, stream),
                SANKHYA_GPU_COPY_FAILED);
    SIH26_QCUDA(cudaStreamSynchronize(stream), SANKHYA_GPU_SYNC_FAILED);
    if (host.state == kDeviceError) throw Failure{SANKHYA_GPU_DEVICE_TIMEOUT, "a grid barrier timed out"};
    if (host.state != kRunning) break;
    if (timed && since() > prm.time_limit) {
      host.state = kTimeLimit;
      break;
    }
    if (steps < 4096) steps *= 2;
  }
  // ---- outputs, un-permuted; the reference's Solution fields (qp_condat_vu.cpp:296-321) ----
  std::vector<double> hx(n), hy(m);
  const int cur = host.cur;
  SIH26_QCUDA(cudaMemcpy(hx.data(), Q.x[cur], n * sizeof(double), cudaMemcpyDeviceToHost), SANKHYA_GPU_COPY_FAILED);
  if (m)
    SIH26_QCUDA(cudaMemcpy(hy.data(), Q.y[cur], m * sizeof(double), cudaMemcpyDeviceToHost), SANKHYA_GPU_COPY_FAILED);
  std::vector<double> x(n), y(m);
  for (int t = 0; t < n; ++t) x[col_perm[t]] = hx[t];
  for (int t = 0; t < m; ++t) y[row_perm[t]] = hy[t];
  for (double v : x)
    if (!std::isfinite(v)) throw Failure{SANKHYA_GPU_NON_FINITE_OUTPUT, "the point is not finite"};
  std::vector<double> qx(n), aty(n, 0.0);
  qp_hessian_multiply(n, hes, x, qx);
  for (int j = 0; j < n; ++j) {
    double dot = 0.0;
    for (int k = prob.col_starts[j]; k < prob.col_starts[j + 1]; ++k) dot += prob.values[k] * y[prob.row_indices[k]];
    aty[j] = dot;
  }
  if (res->col_value) std::memcpy(res->col_value, x.data(), n * sizeof(double));
  if (res->row_dual) for (int i = 0; i < m; ++i) res->row_dual[i] = -sense * y[i];
  if (res->col_dual) for (int j = 0; j < n; ++j) res->col_dual[j] = prob.cost[j] + qx[j] + sense * aty[j];
  // Model::evaluate_objective (src/core/model.cpp:99-125): offset + c'x + 0.5 x'Qx, Q from its
  // lower triangle (an off-diagonal entry counts twice)
  double obj = prob.objective_offset;
  for (int j = 0; j < n; ++j) obj += prob.cost[j] * x[j];
  double quad = 0.0;
  for (int j = 0; j < n; ++j) {
    for (int k = hes.col_starts[j]; k < hes.col_starts[j + 1]; ++k) {
      const int i = hes.row_indices[k];
      quad += (i == j ? 0.5 : 1.0) * hes.values[k] * x[i] * x[j];
    }
  }
  obj += quad;
  res->objective = obj;
  res->converged = host.converged;
  res->iterations = host.iteration;
  res->attempts = host.iteration;
  res->spectral_norm = norm_a;
  std::memset(&res->residuals, 0, sizeof res->residuals);
  res->residuals.absolute_primal = host.best.absolute_primal;
  res->residuals.absolute_dual = host.best.absolute_dual;
  res->residuals.primal_objective = obj;
  // primal_infeasibility: the largest bound violation (Solution::recompute_quality)
  {
    std::vector<double> act(m, 0.0);
    for (int j = 0; j < n; ++j)
      for (int k = prob.col_starts[j]; k < prob.col_starts[j + 1]; ++k) act[prob.row_indices[k]] += prob.values[k] * x[j];
    double worst = 0.0;
    for (int j = 0; j < n; ++j) {
      if (host_finite_bound(prob.col_lower[j])) worst = std::max(worst, prob.col_lower[j] - x[j]);
      if (host_finite_bound(prob.col_upper[j])) worst = std::max(worst, x[j] - prob.col_upper[j]);
    }
    for (int i = 0; i < m; ++i) {
      if (host_finite_bound(prob.row_lower[i])) worst = std::max(worst, prob.row_lower[i] - act[i]);
      if (host_finite_bound(prob.row_upper[i])) worst = std::max(worst, act[i] - prob.row_upper[i]);
    }
    res->primal_infeasibility = worst;
    // the dual measures are the LP engines' (the QP's gradient is c + Qx): not measured here
    res->quality = sankhya_pdhg_quality{worst, NAN, NAN, NAN, NAN, NAN, NAN};
  }
  if (host.state == kConverged) {
    res->status = SANKHYA_PDHG_OPTIMAL;
    std::snprintf(res->message, sizeof res->message,
                  "converged after %lld iterations: primal residual %.3e, dual residual %.3e "
                  "(tolerance %.1e)",
                  host.iteration, host.best.absolute_primal, host.best.absolute_dual, tolerance);
  } else if (host.state == kTimeLimit) {
    res->status = SANKHYA_PDHG_TIME_LIMIT;
    std::snprintf(res->message, sizeof res->message, "time limit %.3gs reached", prm.time_limit);
  } else {
    res->status = SANKHYA_PDHG_ITERATION_LIMIT;
    std::snprintf(res->message, sizeof res->message, "iteration limit %lld reached", c0.iteration_limit);
  }
  res->dual_bound = res->status == SANKHYA_PDHG_OPTIMAL ? obj : (prob.maximize ? INFINITY : -INFINITY);
  res->kernel_launches = launches;
  res->total_seconds = since();
  res->solve_seconds = res->total_seconds;
  return SANKHYA_GPU_SUCCESS;
}

}  // namespace
}  // namespace sih26

extern "C" int sankhya_qp_gpu_solve(const sankhya_pdhg_problem* problem,
                                    const sankhya_qp_hessian* hessian,
                                    const sankhya_pdhg_params* params,
                                    sankhya_pdhg_result* result) {
  using namespace sih26;
  if (!problem || !hessian || !result) {
    g_last_error = "problem, hessian and result must not be NULL";
    return SANKHYA_GPU_INVALID_ARGUMENT;
  }
  sankhya_pdhg_params defaults;
  sankhya_pdhg_gpu_default_params(&defaults);
  if (!params) {
    defaults.tolerance = 1e-8;  // qp_tolerance (src/util/options.cpp:335-341)
    params = &defaults;
  }
  DeviceGuard guard;
  try {
    return qp_solve_impl(*problem, *hessian, *params, result);
  } catch (const Failure& f) {
    g_last_error = f.message;
    std::snprintf(result->message, sizeof result->message, "%s", f.message.c_str());
    result->status = SANKHYA_PDHG_NUMERICAL_ERROR;
    return f.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return SANKHYA_GPU_OUT_OF_MEMORY;
  }
}
