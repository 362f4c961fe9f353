// Batched restarted PDHG: many independent LPs in one persistent launch.
//
// A group of thread blocks -- one block, or a thread-block cluster for the larger LPs --
// takes LPs from a device work queue (largest first) and runs the whole restarted PDHG of
// src/pdhg/pdhg.cpp:267-726 on one LP: the norm estimate, the attempts (phase P, phase D,
// step control), the evaluations every 40 accepted iterations with per-LP restarts and
// termination, and the final report. Phase barriers are __syncthreads for a single block
// and the hardware cluster barrier for a cluster; cluster reductions combine the blocks'
// totals through distributed shared memory in rank order. An LP runs for at most
// `chunk_attempts` attempts per launch and keeps its state in device memory between
// launches, so a host loop can admit and retire LPs between launches.
//
// An LP's work partition is built for its group size alone, so its row sums follow the same
// code and summation order whatever else is in the batch: a result is the same alone and in
// the mix.
//
// Infeasibility and unboundedness: at every evaluation the dual movement since the last
// restart is tested as a Farkas certificate and the last primal step as a primal ray (see
// certificate_test in pdhg_kernels.cuh); the host re-checks every candidate exactly with the
// reference's rules (src/core/certificate.cpp) before reporting it.
#pragma once

#include <cooperative_groups.h>

#include "pdhg_kernels.cuh"

namespace sih26 {

namespace cg = cooperative_groups;

constexpr int kClusterSize = 8;
constexpr long long kChunkNnz = 16384;  // nonzeros per block an attempt of chunk_attempts covers
constexpr int kGroupSlots = 16;

struct BatchSlot {
  Prob<double> P;       // partitions built for the LP's group size
  State<double> S;      // partials and barrier unused
  double* x_out;        // report: unscaled x, permuted
  double* red_out;      // report: min-space reduced costs, permuted
  double* y_out;        // report: unscaled y (PDHG sign), permuted
  double* farkas_out;   // certificate f (reference sign, normalised), permuted
  double* ray_out;      // primal ray r (normalised), permuted
};

// One block.
struct BlockGroup {
  static constexpr int kSize = 1;
  double* red;  // unused
  double* tmp;  // unused
  __device__ __forceinline__ int rank() const { return 0; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
  template <int NS, unsigned MAXMASK>
  __device__ __forceinline__ void reduce(double (&v)[NS], double* sh) const {
    block_reduce<NS, MAXMASK>(v, sh);
  }
  // rank 0's value of a per-block flag, in every block
  __device__ __forceinline__ int agree(int* shared_flag) const {
    __syncthreads();
    return *shared_flag;
  }
};

// A cluster of CS blocks. red[kGroupSlots] and tmp[CS * kGroupSlots] are shared arrays.
template <int CS>
struct ClusterGroup {
  static constexpr int kSize = CS;
  double* red;
  double* tmp;
  __device__ __forceinline__ int rank() const { return (int)cg::this_cluster().block_rank(); }
  __device__ __forceinline__ void sync() const { cg::this_cluster().sync(); }
  template <int NS, unsigned MAXMASK>
  __device__ __forceinline__ void reduce(double (&v)[NS], double* sh) const {
    block_reduce<NS, MAXMASK>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int s = 0; s < NS; ++s) red[s] = v[s];
    }
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    if (threadIdx.x < CS * NS) {
      const int r = threadIdx.x / NS, s = threadIdx.x - r * NS;
      tmp[threadIdx.x] = cl.map_shared_rank(red, r)[s];
    }
    __syncthreads();
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      double t = tmp[s];
      for (int r = 1; r < CS; ++r) {
        const double o = tmp[r * NS + s];
        t = ((MAXMASK >> s) & 1u) ? dmax(t, o) : t + o;
      }
      v[s] = t;
    }
    cl.sync();  // red and tmp are free again
  }
  __device__ __forceinline__ int agree(int* shared_flag) const {
    cg::cluster_group cl = cg::this_cluster();
    cl.sync();
    const int v = *cl.map_shared_rank(shared_flag, 0);
    cl.sync();
    return v;
  }
};

// Norm estimate of the LP's scaled matrix (src/la/scaling.cpp:161-194):
// v = S.xavg holds the random start, u = S.yavg is scratch.
template <class Grp>
__device__ __noinline__ double group_power(const Prob<double>& P, const State<double>& S, int nnz,
                                           double* sh, double* stream, Grp grp) {
  if (P.m == 0 || P.n == 0 || nnz == 0) return 1.0;
  const int rank = grp.rank();
  const int base = rank * kThreads + threadIdx.x, stride = Grp::kSize * kThreads;
  double len2[1] = {0.0};
  for (int j = base; j < P.n; j += stride) {
    const double t = S.xavg[j];
    len2[0] += t * t;
  }
  grp.template reduce<1, 0u>(len2, sh);
  for (int step = 0; step < 30; ++step) {
    const double length = sqrt(len2[0]);
    if (length == 0.0) return 1.0;
    double dummy[1] = {0.0};
    run_phase<1, 1>(P.A.ptr, P.A.idx, P.A.val64, P.pa, ScaledGather{S.xavg, 1.0 / length},
                    StoreRow<1>{S.yavg, -1}, dummy, stream, rank);
    grp.sync();
    double nx[1] = {0.0};
    run_phase<1, 1>(P.AT.ptr, P.AT.idx, P.AT.val64, P.pat, ScaledGather{S.yavg, 1.0},
                    StoreRow<1>{S.xavg, 0}, nx, stream, rank);
    grp.template reduce<1, 0u>(nx, sh);
    len2[0] = nx[0];
  }
  const double norm = sqrt(sqrt(len2[0]));
  return norm > 0.0 ? norm * 1.01 : 1.0;
}

// One evaluation of one LP (pdhg.cpp:502-643) plus the Farkas candidate test. Leaves
// c.state at kRunning, kConverged or kInfeasible.
template <class Grp>
__device__ __noinline__ void group_evaluate(const BatchSlot& B, Ctrl& c, double* sh,
                                            double* stream, int* flags, Grp grp) {
  const Prob<double>& P = B.P;
  const State<double>& S = B.S;
  const int rank = grp.rank();
  const int base = rank * kThreads + threadIdx.x, stride = Grp::kSize * kThreads;
  const int cur = c.cur, prev = cur_prev_slot(c);
  const bool has_average = c.averaged > 0;
  const double count = (double)c.averaged;
  const bool test_cert = c.farkas_cooldown == 0 && (c.evaluations % kCertEvery) == kCertEvery - 1;
  // the Halpern operator's second candidate is the PDHG output T(z_k), not an average
  const bool halpern = c.halpern != 0;
  const double* ray_from = halpern ? S.xt : S.x[cur];
  // E1: running sums and averages, the movement since the last restart (mv) and the
  // certificates' row / column terms (ec, see certificate_test)
  double mv[2] = {0.0, 0.0};
  double ec[kCertSlots];
#pragma unroll
  for (int s = 0; s < kCertSlots; ++s) ec[s] = 0.0;
  for (int j = base; j < P.n; j += stride) {
    const double xo = ld(S.x[cur] + j);
    const double xs = S.xsum[j] + (c.pending ? xo : 0.0);
    S.xsum[j] = xs;
    S.xavg[j] = has_average ? (halpern ? S.xt[j] : xs / count) : 0.0;
    const double d = xo - ld(S.xr + j);
    mv[0] += d * d;
    if (test_cert) {
      const double r = __ldg(P.dc + j) * (ld(ray_from + j) - ld(S.x[prev] + j));
      ray_col_terms(r, __ldg(P.cl0 + j), __ldg(P.cu0 + j), __ldg(P.c0 + j), ec);
    }
  }
  for (int i = base; i < P.m; i += stride) {
    const double yo = ld(S.y[cur] + i);
    const double ys = S.ysum[i] + (c.pending ? yo : 0.0);
    S.ysum[i] = ys;
    S.yavg[i] = has_average ? (halpern ? S.yt[i] : ys / count) : 0.0;
    const double d = yo - ld(S.yr + i);
    mv[1] += d * d;
    if (test_cert) farkas_row_terms(-__ldg(P.dr + i) * d, __ldg(P.rl0 + i), __ldg(P.ru0 + i), ec);
  }
  grp.template reduce<2, 0u>(mv, sh);
  if (test_cert) grp.template reduce<kCertSlots, kCertMaxMask>(ec, sh);
  // E2: residual terms of both candidates (FP64 values)
  double acc[kEvalSlots];
#pragma unroll
  for (int s = 0; s < kEvalSlots; ++s) acc[s] = 0.0;
  RowEval<double, 2> re{P.dr, P.rl0, P.ru0, S.y[cur], S.yavg, nullptr, nullptr};
  run_phase<2, kEvalSlots>(P.A.ptr, P.A.idx, P.A.val64, P.pa,
                           Gather2<double, double>{S.x[cur], S.xavg}, re, acc, stream, rank);
  ColEval<double, 2> ce{P.dc, P.cl0, P.cu0, P.c0, S.x[cur], S.xavg, nullptr, nullptr, nullptr};
  run_phase<2, kEvalSlots>(P.AT.ptr, P.AT.idx, P.AT.val64, P.pat,
                           Gather2<double, double>{S.y[cur], S.yavg}, ce, acc, stream, rank);
  grp.template reduce<kEvalSlots, kEvalMaxMask>(acc, sh);
  // the certificates' matrix terms: A'(y - y_r) and A (x_k - x_{k-1})
  double fk[3] = {0.0, 0.0, 0.0}, rr[2] = {0.0, 0.0};
  if (test_cert) {
    run_phase<1, 3>(P.AT.ptr, P.AT.idx, P.AT.val64, P.pat, DiffGather<double, double>{S.y[cur], S.yr},
                    FarkasCol{P.dc, P.cl0, P.cu0}, fk, stream, rank);
    grp.template reduce<3, kFarkasColMaxMask>(fk, sh);
    run_phase<1, 2>(P.A.ptr, P.A.idx, P.A.val64, P.pa, DiffGather<double, double>{ray_from, S.x[prev]},
                    RayRow{P.dr, P.rl0, P.ru0}, rr, stream, rank);
    grp.template reduce<2, 3u>(rr, sh);
  }
  // every block takes the same decisions from the same totals
  if (threadIdx.x == 0) {
    const Ctrl before = c;
    evaluation_decision(c, acc, mv, has_average, flags);
    flags[3] = 0;
    if (c.farkas_cooldown > 0) --c.farkas_cooldown;
    if (test_cert && c.state != kConverged) {
      const int kind = certificate_test(c, ec, fk, rr);
      if (kind != 0) {
        // keep the restart anchor and step state: the certificate is read from them, and the
        // LP resumes from them if the host turns it down
        const double margin = c.farkas_margin;
        c = before;
        ++c.evaluations;
        c.pending = 0;
        c.farkas_margin = margin;
        c.state = kind == 1 ? kInfeasible : kUnbounded;
        flags[0] = flags[1] = flags[2] = 0;
        flags[3] = kind;
      }
    }
  }
  __syncthreads();
  const double scale = flags[3] == 1 ? ec[1] : ec[3];
  // E3: certificate, best point, restart reset
  if (flags[0] || flags[1] || flags[3]) {
    for (int j = base; j < P.n; j += stride) {
      const double xo = ld(S.x[cur] + j);
      if (flags[3] == 2) B.ray_out[j] = __ldg(P.dc + j) * (ld(ray_from + j) - ld(S.x[prev] + j)) / scale;
      if (flags[0]) S.best_x[j] = flags[2] ? S.xavg[j] : xo;
      if (flags[1]) {
        S.xr[j] = S.x[cur][j];
        S.xsum[j] = 0.0;
      }
    }
    for (int i = base; i < P.m; i += stride) {
      const double yo = ld(S.y[cur] + i);
      if (flags[3] == 1) B.farkas_out[i] = -__ldg(P.dr + i) * (yo - ld(S.yr + i)) / scale;
      if (flags[0]) S.best_y[i] = flags[2] ? S.yavg[i] : yo;
      if (flags[1]) {
        S.yr[i] = S.y[cur][i];
        S.ysum[i] = 0.0;
        if (halpern) S.axr[i] = S.ax[cur][i];  // A x_0 of the new restart point
      }
    }
  }
  grp.sync();
}

// Report of one finished LP (pdhg.cpp:647-661): unscaled point, reduced costs, multipliers
// and the residual block of the best point into c.best.
template <class Grp>
__device__ __noinline__ void group_report(const BatchSlot& B, Ctrl& c, double* sh, double* stream,
                                          Grp grp) {
  const Prob<double>& P = B.P;
  const State<double>& S = B.S;
  const int rank = grp.rank();
  double acc[kEvalSlots];
#pragma unroll
  for (int s = 0; s < kEvalSlots; ++s) acc[s] = 0.0;
  RowEval<double, 1> re{P.dr, P.rl0, P.ru0, nullptr, nullptr, S.best_y, B.y_out};
  run_phase<1, kEvalSlots>(P.A.ptr, P.A.idx, P.A.val64, P.pa, Gather1<double>{S.best_x}, re, acc,
                           stream, rank);
  ColEval<double, 1> ce{P.dc, P.cl0, P.cu0, P.c0, nullptr, nullptr, S.best_x, B.x_out, B.red_out};
  run_phase<1, kEvalSlots>(P.AT.ptr, P.AT.idx, P.AT.val64, P.pat, Gather1<double>{S.best_y}, ce,
                           acc, stream, rank);
  grp.template reduce<kEvalSlots, kReportMaxMask>(acc, sh);
  if (threadIdx.x == 0) {
    c.best = make_residuals(acc, 0, c.bound_norm, c.cost_norm);
    c.primal_violation = dmax(0.0, dmax(acc[1], acc[9]));
  }
  // quality of the reported point (the group's reduction above ordered the outputs' writes)
  double qv[kQualitySlots];
#pragma unroll
  for (int k = 0; k < kQualitySlots; ++k) qv[k] = 0.0;
  quality_pass(P, S.best_x, S.best_y, B.x_out, B.y_out, B.red_out,
               rank * kWarps + (int)(threadIdx.x >> 5), Grp::kSize * kWarps, qv);
  grp.template reduce<kQualitySlots, 0xFFu>(qv, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < kQualitySlots; ++k) c.quality[k] = qv[k];
  }
  __syncthreads();
}

// One attempt of each operator. Inlined: a call per attempt (and the spills of the callee's
// saved registers) cost more than the shared register allocation of the inlined loop.
template <class Grp>
__device__ __forceinline__ void group_halpern_step(const BatchSlot& B, Ctrl& c, double* stream,
                                                   Grp grp) {
  const Prob<double>& P = B.P;
  const State<double>& S = B.S;
  const int rank = grp.rank();
  const int cur = c.cur, nxt = cur ^ 1;
  const double tau = c.eta / c.omega;
  const double sigma = c.eta * c.omega;
  double acc[3] = {0.0, 0.0, 0.0};
  // the Halpern operator (see PrimalStepHalpern in pdhg_kernels.cuh)
  const double w = (double)(c.averaged + 1) / (double)(c.averaged + 2);
  run_phase<1, 3>(P.AT.ptr, P.AT.idx, P.AT.val, P.pat, Gather1<double>{S.y[cur]},
                  PrimalStepHalpern<double>{S.x[cur], S.x[nxt], S.xt, P.c, P.cl, P.cu, S.xr,
                                            tau, w},
                  acc, stream, rank);
  grp.sync();
  run_phase<1, 3>(P.A.ptr, P.A.idx, P.A.val, P.pa, Gather1<double>{S.x[nxt]},
                  DualStepHalpern<double>{S.y[cur], S.y[nxt], S.yt, S.ax[nxt], P.rl, P.ru,
                                          S.yr, S.axr, sigma, w},
                  acc, stream, rank);
  grp.sync();
  if (threadIdx.x == 0) halpern_control(c);
  __syncthreads();
}

template <class Grp>
__device__ __forceinline__ void group_reference_step(const BatchSlot& B, Ctrl& c, double* sh,
                                                     double* stream, Grp grp) {
  const Prob<double>& P = B.P;
  const State<double>& S = B.S;
  const int rank = grp.rank();
  const int cur = c.cur, nxt = cur ^ 1;
  const double tau = c.eta / c.omega;
  const double sigma = c.eta * c.omega;
  double acc[3] = {0.0, 0.0, 0.0};
  {
    PrimalStep<double> ps{S.x[cur], S.x[nxt], P.c, P.cl, P.cu, S.xsum, tau, c.pending};
    run_phase<1, 3>(P.AT.ptr, P.AT.idx, P.AT.val, P.pat, Gather1<double>{S.y[cur]}, ps, acc,
                    stream, rank);
  }
  grp.sync();
  {
    DualStep<double> ds{S.y[cur], S.y[nxt], S.ax[cur], S.ax[nxt], P.rl, P.ru, S.ysum, sigma,
                        c.pending};
    run_phase<1, 3>(P.A.ptr, P.A.idx, P.A.val, P.pa, Gather1<double>{S.x[nxt]}, ds, acc,
                    stream, rank);
  }
  grp.template reduce<3, 0u>(acc, sh);
  if (threadIdx.x == 0) step_control(c, acc);
  __syncthreads();
}

template <class Grp>
__device__ inline void run_instance(const BatchSlot& B, Ctrl& c, double* sh, double* stream,
                                    int* flags, long long chunk_attempts, Grp grp) {
  const Prob<double>& P = B.P;
  const State<double>& S = B.S;
  const int rank = grp.rank();
  if (threadIdx.x == 0) c = *S.ctrl;
  __syncthreads();
  // The chunk is a budget of work, not of attempts: chunk_attempts for an LP with at most
  // kChunkNnz nonzeros per block, proportionally fewer attempts (at least 8) for larger ones,
  // so a launch lasts about as long for every LP and no slot idles behind one large LP.
  {
    const long long per_block = (long long)__ldg(P.A.ptr + P.m) / Grp::kSize;
    if (per_block > kChunkNnz && chunk_attempts < (1ll << 40)) {
      const long long scaled = chunk_attempts * kChunkNnz / per_block;
      chunk_attempts = scaled < 8 ? 8 : scaled;
    }
  }
  if (c.state == kSetup) {
    const int nnz = __ldg(P.A.ptr + P.m);
    const double norm = group_power(P, S, nnz, sh, stream, grp);
    if (threadIdx.x == 0) {
      c.spectral_norm = norm;
      c.eta = norm > 0.0 ? 1.0 / norm : 1.0;
      if (c.halpern) c.eta = 0.998 / dmax(norm, 1e-12);  // constant: tau sigma ||A||^2 < 1
      c.eta_ceiling = 1.0e3 / dmax(norm, 1e-12);
      c.state = kRunning;
    }
    double dummy[1] = {0.0};
    run_phase<1, 1>(P.A.ptr, P.A.idx, P.A.val, P.pa, Gather1<double>{S.x[0]},
                    StoreRow<1>{S.ax[0], -1}, dummy, stream, rank);
    grp.sync();
    if (c.halpern) {  // A x_0 of the starting point
      const int base = rank * kThreads + threadIdx.x, stride = Grp::kSize * kThreads;
      for (int i = base; i < P.m; i += stride) S.axr[i] = S.ax[0][i];
      grp.sync();
    }
  }
  long long a = 0;
  while (c.state == kRunning) {
    // loop top (pdhg.cpp:384-385); the deadline is read by rank 0 and agreed on
    const bool check_clock = c.deadline_ns != 0ull && (a & 63) == 0;
    if (threadIdx.x == 0) {
      flags[5] = 0;
      flags[6] = (check_clock && global_ns() > c.deadline_ns) ? 1 : 0;
      if (c.iteration >= c.iteration_limit) {
        c.state = kIterationLimit;
      } else if (a >= chunk_attempts) {
        flags[5] = 1;
      }
    }
    if (check_clock) {
      const int late = grp.agree(&flags[6]);
      if (late && threadIdx.x == 0 && c.state == kRunning) c.state = kTimeLimit;
    }
    __syncthreads();
    if (c.state != kRunning || flags[5]) break;
    ++a;
    if (c.halpern) group_halpern_step(B, c, stream, grp);
    else group_reference_step(B, c, sh, stream, grp);
    if (c.state == kNeedEval) group_evaluate(B, c, sh, stream, flags, grp);
  }
  if (c.state == kConverged || c.state == kIterationLimit || c.state == kTimeLimit ||
      c.state == kInfeasible || c.state == kUnbounded) {
    group_report(B, c, sh, stream, grp);
  }
  if (threadIdx.x == 0 && rank == 0) *S.ctrl = c;
  grp.sync();
}

// The persistent batch kernels: blocks (or clusters) take LPs from the active list through a
// device counter (the list is ordered largest first) until it is exhausted.
__global__ void __launch_bounds__(kThreads, 2) batch_kernel(const BatchSlot* slots,
                                                            const int* active,
                                                            const int* active_count,
                                                            int* queue_head,
                                                            long long chunk_attempts) {
  __shared__ Ctrl c;
  __shared__ double sh[kWarps * kEvalSlots];
  __shared__ int flags[8];
  __shared__ int s_take;
  double* stream = warp_stream();
  const int count = *active_count;
  for (;;) {
    if (threadIdx.x == 0) s_take = atomicAdd(queue_head, 1);
    __syncthreads();
    const int q = s_take;
    __syncthreads();
    if (q >= count) break;
    run_instance(slots[active[q]], c, sh, stream, flags, chunk_attempts,
                 BlockGroup{nullptr, nullptr});
  }
}

__global__ void __cluster_dims__(kClusterSize, 1, 1) __launch_bounds__(kThreads, 2)
    cluster_batch_kernel(const BatchSlot* slots, const int* active, const int* active_count,
                         int* queue_head, long long chunk_attempts) {
  __shared__ Ctrl c;
  __shared__ double sh[kWarps * kEvalSlots];
  __shared__ double red[kGroupSlots];
  __shared__ double tmp[kClusterSize * kGroupSlots];
  __shared__ int flags[8];
  __shared__ int s_take;
  double* stream = warp_stream();
  const ClusterGroup<kClusterSize> grp{red, tmp};
  cg::cluster_group cl = cg::this_cluster();
  const int count = *active_count;
  for (;;) {
    if (cl.block_rank() == 0 && threadIdx.x == 0) s_take = atomicAdd(queue_head, 1);
    cl.sync();
    const int q = *cl.map_shared_rank(&s_take, 0);
    cl.sync();
    if (q >= count) break;
    run_instance(slots[active[q]], c, sh, stream, flags, chunk_attempts, grp);
  }
}

// Copies the control blocks of the active LPs into one compact array for the host.
__global__ void gather_ctrl_kernel(const Ctrl* ctrls, const int* active, const int* active_count,
                                   Ctrl* out) {
  const int count = *active_count;
  for (int q = blockIdx.x; q < count; q += gridDim.x) {
    const int* src = reinterpret_cast<const int*>(ctrls + active[q]);
    int* dst = reinterpret_cast<int*>(out + q);
    for (int w = threadIdx.x; w < (int)(sizeof(Ctrl) / sizeof(int)); w += blockDim.x) dst[w] = src[w];
  }
}

}  // namespace sih26
