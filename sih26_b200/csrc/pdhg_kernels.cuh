// Restarted-PDHG kernels for sm_100a.
//
// Iteration = src/pdhg/pdhg.cpp:383-644 restructured for one GPU:
//
//   iterate_kernel (cooperative, persistent over a chunk of attempts)
//     phase P  (rows of A' = columns of A, resident CSR of A'):
//              g_j = (A' y)_j, x'_j = proj(x_j - tau (c_j + g_j)), partial sum of (x'-x)^2,
//              and the running sum x_sum += x for the iterate accepted last attempt
//     barrier
//     phase D  (rows of A, resident CSR of A):
//              a'_i = (A x')_i, abar = 2 a' - a, adx = a' - a   (a = A x kept from the
//              accepted iterate: one SpMV gives both A xbar and A dx, pdhg.cpp:403,432),
//              y'_i = v - sigma proj(v / sigma, [rl, ru]), v = y + sigma abar,
//              partial sums of (y'-y)^2 and (y'-y) adx, and y_sum += y
//     barrier
//     control  every block reduces the same partials in the same order, so every block
//              takes the same accept / step-size decision (pdhg.cpp:413-496) without
//              another barrier
//   evaluate_kernel (cooperative), after every 40th accepted iteration or a step without
//     information (pdhg.cpp:502-503): unscaled FP64 residuals of the current iterate and of
//     the running average (pdhg.cpp:143-263), candidate choice, best point, stopping test
//     and restart with the primal-weight update (pdhg.cpp:505-643).
//   report_kernel: the best point in original units, its residuals and its quality block
//     (Solution::recompute_quality, src/core/model.cpp:228-424).
//
// The iteration kernel has one instance per operator: the reference's adaptive step above,
// and the reflected Halpern step (PrimalStepHalpern below: a constant step, no acceptance
// test, the second candidate is the PDHG output T(z) instead of the average).
//
// Two precision levels share this code: FP64 (iterates, matrix and reductions in FP64) and
// the FP32 level of the mixed mode (FP32 matrix and FP32 iterate deltas about an FP64 restart
// anchor, FP64 accumulation; see kDelta), which hands over to FP64 only if it stops improving.
//
// Internal index spaces are permuted: rows of A sorted by nonzero count (descending) and
// columns likewise, so a work item holds rows of similar length; the host un-permutes
// outputs. Reductions use fixed trees over a fixed work partition, so a run is bit-for-bit
// repeatable; the Halpern phases, which reduce nothing, let a block's warps share its items
// at run time (each row is still summed by one warp in a fixed order).
#pragma once

#include <cstdint>
#include <type_traits>

#include "device_common.cuh"

namespace sih26 {

// Solver states (Ctrl::state).
enum : int {
  kRunning = 0,
  kNeedEval = 1,
  kConverged = 2,
  kIterationLimit = 3,
  kTimeLimit = 4,
  kDeviceError = 5,
  kSetup = 6,       // batched LPs: norm estimate and A x0 still to do
  kInfeasible = 7,  // a Farkas certificate passed the device test (the host re-checks it)
  kUnbounded = 8    // a primal ray passed the device test (the host re-checks it)
};

struct Residuals {
  double primal, dual, gap, primal_objective, dual_objective, absolute_primal, absolute_dual,
      gap_as_verified, complementarity;
};

// Quality of a reported point (Solution::recompute_quality, src/core/model.cpp:228-424), every
// slot a maximum of non-negative terms: 0 primal_infeasibility, 1 primal_infeasibility_scaled,
// 2 dual_infeasibility, 3 dual_infeasibility_scaled (column terms), 4
// complementarity_violation, 5 the largest row-price sign violation and 6 the largest row
// complementarity product over its row scale (both divided by the dual-norm scale once slot 7,
// max |row_dual|, is known).
constexpr int kQualitySlots = 8;

// Host <-> device control block of one LP. Block 0 writes it at kernel exit; every block
// reads it at kernel entry.
struct Ctrl {
  // step state
  double eta, omega, restart_kkt, best_worst;
  long long iteration, attempts, averaged, last_restart, restarts, evaluations;
  int cur, pending, state, converged;
  int chosen_average, best_is_set, pad0, halpern;  // halpern: the Halpern operator
  Residuals best, current, average;  // best so far; last evaluation's two candidates
  // constants of the solve
  double spectral_norm, eta_ceiling, tolerance, bound_norm, cost_norm;
  long long iteration_limit;
  int use_restarts, stop_at_request, stop_rule, pad2;
  int time_up, farkas_cooldown;
  unsigned long long deadline_ns;  // batched LPs: device-clock deadline, 0 = none
  double farkas_margin;            // batched LPs: normalised margin S - M of the last test
  double primal_violation;         // report: the reported point's largest bound violation
  double quality[kQualitySlots];   // report: the reported point's quality slots (above)
};

// SpMV work partition of one CSR matrix in permuted row order (rows sorted by length,
// longest first). Per block b:
//   segments  [blk_seg_begin[b], +1): {row, nz_begin, nz_end, 0}, pieces of <= kSegment
//             nonzeros of this block's long rows (> kItemNnz nonzeros), one warp each;
//   long rows [blk_long_begin[b], +1): {row, first segment, segments, 0}; once the block's
//             segments are done, a warp sums a long row's segment partials in order and
//             runs the row's epilogue;
//   items     [blk_item_begin[b], +1): {row_begin, row_end, lanes, 0}:
//             lanes == 0: a stream item, <= 32 rows of <= kStreamRowMax nonzeros and
//               <= kItemNnz in total; the warp loads all of it at once, parks the products
//               in shared memory, then lane r sums row r in order and runs its epilogue;
//             lanes > 0: 32/lanes rows of up to kItemNnz nonzeros, one group of `lanes`
//               lanes per row, reduced by shuffles.
// Every long row lives in one block, so no partial crosses blocks and no atomics are needed.
constexpr int kSegment = 512;
constexpr int kItemNnz = 512;
constexpr int kStreamRowMax = 32;

struct Part {
  const int* blk_seg_begin;
  const int4* segs;
  const int* blk_long_begin;
  const int4* longs;
  const int* blk_item_begin;
  const int4* items;
  double* seg_sum;  // [segments * 2] scratch
  // sliced partitions only (the iteration kernel's): the slice arrays, column indices and
  // values (of the level's value type) in slice order; items {row_begin, row_end, -L, offset}
  const int* sell_idx;
  const void* sell_val;
};

// Unrolled loads per lane and round in a slice: every round issues this many independent
// gathers before it sums them (4 measured fastest of 4, 6, 8, 12 and 16 on the 5M-nonzero LP:
// fewer dead slots on short rows, fewer registers).
constexpr int kSliceUnroll = 4;

template <class T>
struct Csr {
  const int* ptr;
  const int* idx;
  const T* val;
  const double* val64;  // FP64 values (== val when T is double)
};

template <class T>
struct Prob {
  int m, n;
  Csr<T> A, AT;
  Part pa, pat;
  Part pai, pati;  // the iteration kernel's sliced partitions (slice values of type T)
  Part pae, pate;  // the evaluation's: the same slices with FP64 values (the FP64 level's)
  // scaled problem, permuted (src/la/scaling.hpp:36-58)
  const T* c;
  const T* cl;
  const T* cu;
  const T* rl;
  const T* ru;
  // the same in FP64 (the FP32 level projects and forms its anchor terms with these)
  const double* c64;
  const double* cl64;
  const double* cu64;
  const double* rl64;
  const double* ru64;
  const double* dr;  // row scaling Dr, permuted
  const double* dc;  // column scaling Dc, permuted
  // unscaled problem, permuted; c0 is the min-space cost (pdhg.cpp:287-291)
  const double* c0;
  const double* cl0;
  const double* cu0;
  const double* rl0;
  const double* ru0;
};

template <class T>
struct State {
  // FP64 level: x, y are the iterates and ax = A x. FP32 level: x, y are FP32 deltas from the
  // FP64 restart anchor (xr, yr), ax = A dx, and xsum, ysum sum the deltas (see kDelta).
  T* x[2];
  T* y[2];
  double* ax[2];
  double* xsum;
  double* ysum;
  double* xr;  // restart anchor
  double* yr;
  // FP32 level only: the anchor's terms, refreshed at every restart
  double* cg;     // [n] c + A'yr (scaled)
  float* dl;      // [n] lower bound - xr, rounded to FP32
  float* du;      // [n] upper bound - xr
  double* axr;    // [m] A xr (the Halpern operator needs it on the FP64 level too)
  T* xt;          // Halpern: the PDHG output T(z_k), primal part (a delta on the FP32 level)
  T* yt;          // and dual part
  double* xavg;   // [n] batched engine: the evaluation's second candidate
  double* yavg;   // [m]
  // single-LP evaluation: both candidates of every column / row side by side (the current
  // point in FP64, then the second candidate), so one 16-byte gather reads both
  double2* xc;  // [n]
  double2* yc;  // [m]
  double* best_x;  // scaled, FP64
  double* best_y;
  double* cert_row;  // [m] Farkas candidate (reference sign, max-normalised), permuted
  double* cert_col;  // [n] primal-ray candidate (max-normalised), permuted
  double* partials;  // [2][G][kPartSlots]
  Ctrl* ctrl;
  GridBarrier bar;
};

constexpr int kPartSlots = 32;
constexpr int kEvalSlots = 16;
// complementarity slots of the evaluation are max-reductions
constexpr unsigned kEvalMaxMask = (1u << 6) | (1u << 7) | (1u << 12) | (1u << 13);
// the report (one candidate) also keeps the largest row and column bound violations of the
// point in the second candidate's slots 1 and 9: Solution::recompute_quality's
// primal_infeasibility (src/core/model.cpp:228-283), on the device
constexpr unsigned kReportMaxMask = kEvalMaxMask | (1u << 1) | (1u << 9);

// dynamic shared memory of the phase kernels: one stream buffer of kItemNnz products per warp
constexpr size_t stream_smem_bytes() { return (size_t)kWarps * kItemNnz * sizeof(double); }

// Loads of iterate vectors written earlier in the same launch by other blocks. Plain
// (L1-cacheable) loads: the grid barrier's release/acquire pairs order them after the
// writes, and L1 keeps the hot entries of a gathered vector close.
template <class T>
__device__ __forceinline__ double ld(const T* p) {
  return static_cast<double>(*p);
}

__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Pulls a contiguous nonzero range [nz0, nz1) of one CSR matrix towards L2, one 128-byte line
// per lane per step.
template <class V>
__device__ __forceinline__ void prefetch_range(const int* idx, const V* val, int nz0, int nz1,
                                               int lane) {
  for (int k = nz0 + lane * 32; k < nz1; k += 32 * 32) prefetch_l2(idx + k);
  constexpr int per_line = 128 / (int)sizeof(V);
  for (int k = nz0 + lane * per_line; k < nz1; k += 32 * per_line) prefetch_l2(val + k);
}
template <class T>
__device__ __forceinline__ double ro(const T* p) {
  return static_cast<double>(__ldg(p));
}


// Streamed matrix loads of the sliced phases (the iteration kernel's): each entry is read once
// per phase, so they bypass L1 (no_allocate) and leave it to the gathered vector.
__device__ __forceinline__ int ld_stream(const int* p) {
  int v;
  asm("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ float ld_stream(const float* p) {
  float v;
  asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ double ld_stream(const double* p) {
  double v;
  asm("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(p));
  return v;
}

// Whether a gather reads its NV vectors with one load (GatherPair).
template <class G, class = void>
struct paired_gather : std::false_type {};
template <class G>
struct paired_gather<G, std::void_t<decltype(G::kPaired)>> : std::bool_constant<G::kPaired> {};

// ---- generic fused SpMV phase ----------------------------------------------------------
//
// For every row r of the matrix owned by this block: s = sum_k val[k] * gather(idx[k])
// (NV gathered vectors at once, FP64 accumulation), then the epilogue:
//   typename Epi::In in = epi.load(r);   issued before the row's sum so its loads overlap
//   epi.apply(r, s, in, acc);
// `stream` is this warp's kItemNnz doubles of dynamic shared memory; a stream item with
// NV > 1 gathered vectors passes over it once per vector.
//
// kShared: the block's warps take its short-row items from a shared-memory counter as they
// finish the last one, instead of every 16th item each, so no warp idles while another still
// has two items to go. For phases that reduce nothing across rows: a row's sum is the same
// whichever warp takes it, but a per-thread accumulator would group its terms differently.
//
// kSliced: the partition holds slices instead of stream items (partition(..., sliced = true)):
// lane l of the warp owns row row_begin + l and sums it in its stored order from the slice
// arrays, kUnroll independent gathers in flight per round; the products are summed in the
// row's order, as in a stream item. Such a phase uses no shared-memory stream buffer.
//
// kLateIn: slices and grouped rows load the epilogue's inputs after the row's sum instead of
// before it, so they hold no registers during the sum (for epilogues with many inputs).
template <int NV, int NS, bool kShared = false, bool kSliced = false, int kUnroll = kSliceUnroll,
          bool kLateIn = false, class V, class Gather, class Epi>
__device__ __forceinline__ void run_phase(const int* __restrict__ ptr, const int* __restrict__ idx,
                                          const V* __restrict__ val, const Part& p,
                                          const Gather& g, const Epi& epi, double (&acc)[NS],
                                          double* stream, int blk = -1) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int b = blk >= 0 ? blk : (int)blockIdx.x;
  // 1. segments of long rows: one warp per segment
  const int sb = __ldg(p.blk_seg_begin + b), se = __ldg(p.blk_seg_begin + b + 1);
  for (int q = sb + warp; q < se; q += kWarps) {
    const int4 sg = __ldg(p.segs + q);
    double s[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] = 0.0;
#pragma unroll
    for (int t = 0; t < kSegment / 32; ++t) {
      const int k = sg.y + lane + 32 * t;
      if (k < sg.z) {
        if constexpr (kSliced)
          g.add(s, static_cast<double>(ld_stream(val + k)), ld_stream(idx + k));
        else
          g.add(s, ro(val + k), __ldg(idx + k));
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
      for (int v = 0; v < NV; ++v) s[v] += __shfl_xor_sync(0xffffffffu, s[v], off);
    }
    if (lane == 0) {
#pragma unroll
      for (int v = 0; v < NV; ++v) p.seg_sum[(size_t)q * NV + v] = s[v];
    }
  }
  // 2. short rows; each item first pulls the warp's next item towards L2
  const int ib = __ldg(p.blk_item_begin + b), ie = __ldg(p.blk_item_begin + b + 1);
  __shared__ int next_item;  // kShared: the block's next unclaimed item
  if constexpr (kShared) {
    if (threadIdx.x == 0) next_item = ib + kWarps;  // the first kWarps go one to each warp
    __syncthreads();
  }
  int4 item = ib + warp < ie ? __ldg(p.items + ib + warp) : make_int4(0, 0, 0, 0);
  for (int it = ib + warp; it < ie;) {
    int4 next = make_int4(0, 0, 0, 0);
    int nit;
    if constexpr (kShared) {
      nit = lane == 0 ? atomicAdd(&next_item, 1) : 0;
      nit = __shfl_sync(0xffffffffu, nit, 0);
    } else {
      nit = it + kWarps;
    }
    if (nit < ie) {
      next = __ldg(p.items + nit);
      if (kSliced && next.z < 0)
        prefetch_range(p.sell_idx, static_cast<const V*>(p.sell_val), next.w,
                       next.w + (next.y - next.x) * (-next.z), lane);
      else
        prefetch_range(idx, val, __ldg(ptr + next.x), __ldg(ptr + next.y), lane);
    }
    if (kSliced && item.z < 0) {
      if constexpr (kSliced) {
        // slice: lane l sums row item.x + l over the slice arrays
        const int rows = item.y - item.x, L = -item.z;
        const int r = item.x + lane;
        const bool mine = lane < rows;
        typename Epi::In in{};
        int len = 0;
        if (mine) {
          if constexpr (!kLateIn) in = epi.load(r);
          len = __ldg(ptr + r + 1) - __ldg(ptr + r);
        }
        const int* __restrict__ si = p.sell_idx + item.w + lane;
        const V* __restrict__ sv = static_cast<const V*>(p.sell_val) + item.w + lane;
        double s[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) s[v] = 0.0;
        // values and gathered entries stay in their stored width until the multiply; a
        // product of two FP32 numbers is exact in FP64, so the sum is the stream item's.
        // FP32 slices load the next round's column indices while this round's entries are
        // gathered (kPipe; measured faster there, slower with FP64 values).
        constexpr bool kPipe = sizeof(V) == 4;
        int jn[kUnroll];
        if constexpr (kPipe) {
#pragma unroll
          for (int t = 0; t < kUnroll; ++t)
            jn[t] = (mine && t < len) ? ld_stream(si + (size_t)t * rows) : 0;
        }
        for (int k0 = 0; k0 < L; k0 += kUnroll) {
          int j[kUnroll];
          V a[kUnroll];
#pragma unroll
          for (int t = 0; t < kUnroll; ++t) {
            const bool live = mine && k0 + t < len;
            if constexpr (kPipe)
              j[t] = jn[t];
            else
              j[t] = live ? ld_stream(si + (size_t)(k0 + t) * rows) : 0;
            a[t] = live ? ld_stream(sv + (size_t)(k0 + t) * rows) : V(0);
          }
          if constexpr (kPipe) {
#pragma unroll
            for (int t = 0; t < kUnroll; ++t) {
              const int k = k0 + kUnroll + t;
              jn[t] = (mine && k < len) ? ld_stream(si + (size_t)k * rows) : 0;
            }
          }
          if constexpr (paired_gather<Gather>::value) {
            static_assert(NV == 2, "a paired gather reads two vectors");
            double2 gv[kUnroll];
#pragma unroll
            for (int t = 0; t < kUnroll; ++t)
              gv[t] = (mine && k0 + t < len) ? g.pair(j[t]) : make_double2(0.0, 0.0);
#pragma unroll
            for (int t = 0; t < kUnroll; ++t)
              if (k0 + t < len) {
                s[0] += static_cast<double>(a[t]) * gv[t].x;
                s[1] += static_cast<double>(a[t]) * gv[t].y;
              }
          } else {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              typename Gather::Raw gv[kUnroll];
#pragma unroll
              for (int t = 0; t < kUnroll; ++t)
                gv[t] = (mine && k0 + t < len) ? g.raw(v, j[t]) : typename Gather::Raw(0);
#pragma unroll
              for (int t = 0; t < kUnroll; ++t)
                if (k0 + t < len) s[v] += static_cast<double>(a[t]) * static_cast<double>(gv[t]);
            }
          }
        }
        if (mine) {
          if constexpr (kLateIn) in = epi.load(r);
          epi.apply(r, s, in, acc);
        }
      }
    } else if (kSliced && item.z == 0) {
      // never produced by a sliced partition
    } else if (!kSliced && item.z == 0) {
      // stream item
      const int rows = item.y - item.x;
      const int r = item.x + lane;
      const bool mine = lane < rows;
      typename Epi::In in{};
      int rb = 0, re = 0;
      if (mine) {
        in = epi.load(r);
        rb = __ldg(ptr + r);
        re = __ldg(ptr + r + 1);
      }
      const int nz0 = __ldg(ptr + item.x), nz1 = __ldg(ptr + item.y);
      double s[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
#pragma unroll
        for (int t = 0; t < kItemNnz / 32; ++t) {
          const int k = nz0 + lane + 32 * t;
          if (k < nz1) stream[k - nz0] = g.product(v, ro(val + k), __ldg(idx + k));
        }
        __syncwarp();
        double sum = 0.0;
        if (mine) {
          for (int k = rb - nz0; k < re - nz0; ++k) sum += stream[k];
        }
        s[v] = sum;
        __syncwarp();
      }
      if (mine) epi.apply(r, s, in, acc);
    } else {
      // grouped item: one group of item.z lanes per row
      const int lanes = item.z;
      const int gid = lane / lanes, gl = lane - gid * lanes;
      const int r = item.x + gid;
      const bool valid = r < item.y;
      typename Epi::In in{};
      double s[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) s[v] = 0.0;
      if (valid) {
        if (!kLateIn && gl == 0) in = epi.load(r);
        const int kb = __ldg(ptr + r), ke = __ldg(ptr + r + 1);
        if constexpr (kSliced) {
          // the lane's entries kb + gl, kb + gl + lanes, ... in rounds of kUnroll independent
          // raw-width gathers, summed in that same order (so the sums are those of the plain
          // loop below, bit for bit)
          // FP32 values: the next round's column indices are loaded while this round's
          // entries are gathered, as in a slice
          constexpr bool kPipe = sizeof(V) == 4;
          int jn[kUnroll];
          if constexpr (kPipe) {
#pragma unroll
            for (int t = 0; t < kUnroll; ++t) {
              const int k = kb + gl + t * lanes;
              jn[t] = k < ke ? ld_stream(idx + k) : 0;
            }
          }
          for (int k0 = kb + gl; k0 < ke; k0 += lanes * kUnroll) {
            int j[kUnroll];
            V a[kUnroll];
#pragma unroll
            for (int t = 0; t < kUnroll; ++t) {
              const int k = k0 + t * lanes;
              if constexpr (kPipe)
                j[t] = jn[t];
              else
                j[t] = k < ke ? ld_stream(idx + k) : 0;
              a[t] = k < ke ? ld_stream(val + k) : V(0);
            }
            if constexpr (kPipe) {
#pragma unroll
              for (int t = 0; t < kUnroll; ++t) {
                const int k = k0 + (kUnroll + t) * lanes;
                jn[t] = k < ke ? ld_stream(idx + k) : 0;
              }
            }
            if constexpr (paired_gather<Gather>::value) {
              double2 gv[kUnroll];
#pragma unroll
              for (int t = 0; t < kUnroll; ++t)
                gv[t] = k0 + t * lanes < ke ? g.pair(j[t]) : make_double2(0.0, 0.0);
#pragma unroll
              for (int t = 0; t < kUnroll; ++t)
                if (k0 + t * lanes < ke) {
                  s[0] += static_cast<double>(a[t]) * gv[t].x;
                  s[1] += static_cast<double>(a[t]) * gv[t].y;
                }
            } else {
#pragma unroll
              for (int v = 0; v < NV; ++v) {
                typename Gather::Raw gv[kUnroll];
#pragma unroll
                for (int t = 0; t < kUnroll; ++t)
                  gv[t] = k0 + t * lanes < ke ? g.raw(v, j[t]) : typename Gather::Raw(0);
#pragma unroll
                for (int t = 0; t < kUnroll; ++t)
                  if (k0 + t * lanes < ke)
                    s[v] += static_cast<double>(a[t]) * static_cast<double>(gv[t]);
              }
            }
          }
        } else {
#pragma unroll 16
          for (int k = kb + gl; k < ke; k += lanes) g.add(s, ro(val + k), __ldg(idx + k));
        }
      }
      for (int off = lanes >> 1; off > 0; off >>= 1) {
#pragma unroll
        for (int v = 0; v < NV; ++v) s[v] += __shfl_xor_sync(0xffffffffu, s[v], off);
      }
      if (valid && gl == 0) {
        if constexpr (kLateIn) in = epi.load(r);
        epi.apply(r, s, in, acc);
      }
    }
    item = next;
    it = nit;
  }
  // 3. long rows: sum the block's segment partials in segment order, then the epilogue
  const int lb = __ldg(p.blk_long_begin + b), le = __ldg(p.blk_long_begin + b + 1);
  if (le > lb) {
    __syncthreads();
    for (int q = lb + warp; q < le; q += kWarps) {
      const int4 lr = __ldg(p.longs + q);
      typename Epi::In in{};
      if (lane == 0) in = epi.load(lr.x);
      double s[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) s[v] = 0.0;
      for (int k = lane; k < lr.z; k += 32) {
#pragma unroll
        for (int v = 0; v < NV; ++v) s[v] += p.seg_sum[(size_t)(lr.y + k) * NV + v];
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int v = 0; v < NV; ++v) s[v] += __shfl_xor_sync(0xffffffffu, s[v], off);
      }
      if (lane == 0) epi.apply(lr.x, s, in, acc);
    }
  }
}

// ---- gathers -------------------------------------------------------------------------

template <class T>
struct Gather1 {
  const T* v;
  using Raw = T;  // the gathered entry as stored (sliced phases)
  __device__ __forceinline__ void add(double (&s)[1], double a, int k) const { s[0] += a * ld(v + k); }
  __device__ __forceinline__ double product(int, double a, int k) const { return a * ld(v + k); }
  __device__ __forceinline__ T raw(int, int k) const { return v[k]; }
};

template <class T, class U>
struct Gather2 {
  const T* v0;
  const U* v1;
  __device__ __forceinline__ void add(double (&s)[2], double a, int k) const {
    s[0] += a * ld(v0 + k);
    s[1] += a * ld(v1 + k);
  }
  __device__ __forceinline__ double product(int which, double a, int k) const {
    return which == 0 ? a * ld(v0 + k) : a * ld(v1 + k);
  }
};

// Two FP64 vectors stored side by side: one 16-byte load gathers both entries. Each sum is
// formed in the same order as with two separate gathers (Gather2), so the sums are the same.
struct GatherPair {
  const double2* v;
  static constexpr bool kPaired = true;
  __device__ __forceinline__ void add(double (&s)[2], double a, int k) const {
    const double2 t = v[k];
    s[0] += a * t.x;
    s[1] += a * t.y;
  }
  __device__ __forceinline__ double product(int which, double a, int k) const {
    const double2 t = v[k];
    return a * (which == 0 ? t.x : t.y);
  }
  __device__ __forceinline__ double2 pair(int k) const { return v[k]; }
};


// ---- epilogues of the iteration ---------------------------------------------------------

// x' = proj_X(x - tau (c + A'y))  (pdhg.cpp:392-400); slot 0 gets (x'-x)^2.
template <class T>
struct PrimalStep {
  const T* x;
  T* xn;
  const T* c;
  const T* cl;
  const T* cu;
  double* xsum;
  double tau;
  int pending;
  struct In {
    double xo, c, lo, hi, xs;
  };
  __device__ __forceinline__ In load(int j) const {
    In v;
    v.xo = ld(x + j);
    v.c = ro(c + j);
    v.lo = ro(cl + j);
    v.hi = ro(cu + j);
    v.xs = pending ? __ldcg(xsum + j) : 0.0;
    return v;
  }
  __device__ __forceinline__ void apply(int j, const double (&s)[1], const In& v,
                                        double (&acc)[3]) const {
    if (pending) xsum[j] = v.xs + v.xo;
    const double xnew = project(v.xo - tau * (v.c + s[0]), v.lo, v.hi);
    const T xs = static_cast<T>(xnew);
    xn[j] = xs;
    const double d = static_cast<double>(xs) - v.xo;
    acc[0] += d * d;
  }
};

// y' = v - sigma proj_C(v / sigma), v = y + sigma A xbar  (pdhg.cpp:402-408);
// slots 1, 2 get (y'-y)^2 and (y'-y) (A dx)_i.
template <class T>
struct DualStep {
  const T* y;
  T* yn;
  const double* ax;
  double* axn;
  const T* rl;
  const T* ru;
  double* ysum;
  double sigma;
  int pending;
  struct In {
    double yo, aold, lo, hi, ys;
  };
  __device__ __forceinline__ In load(int i) const {
    In v;
    v.yo = ld(y + i);
    v.aold = __ldcg(ax + i);
    v.lo = ro(rl + i);
    v.hi = ro(ru + i);
    v.ys = pending ? __ldcg(ysum + i) : 0.0;
    return v;
  }
  __device__ __forceinline__ void apply(int i, const double (&s)[1], const In& v,
                                        double (&acc)[3]) const {
    if (pending) ysum[i] = v.ys + v.yo;
    const double anew = s[0];
    const double w = v.yo + sigma * (2.0 * anew - v.aold);
    const double ynew = w - sigma * project(w / sigma, v.lo, v.hi);
    const T ys = static_cast<T>(ynew);
    yn[i] = ys;
    axn[i] = anew;
    const double d = static_cast<double>(ys) - v.yo;
    acc[1] += d * d;
    acc[2] += d * (anew - v.aold);
  }
};

// Stores the row sum (setup of A x0, and the power iteration); optionally its square.
template <int NS>
struct StoreRow {
  double* out;
  int square_into;  // slot that gets s^2, or -1
  struct In {};
  __device__ __forceinline__ In load(int) const { return In{}; }
  __device__ __forceinline__ void apply(int r, const double (&s)[1], const In&, double (&acc)[NS]) const {
    out[r] = s[0];
    if (square_into >= 0) acc[square_into] += s[0] * s[0];
  }
};

// ---- the FP32 level: deltas from an FP64 restart anchor ---------------------------------
//
// The FP32 level keeps x = xr + dx and y = yr + dy with the anchor (xr, yr) in FP64 and the
// deltas in FP32. The anchor's terms are formed once per restart in FP64 (cg = c + A'yr,
// axr = A xr, bounds relative to xr), so each iteration streams the FP32 matrix and gathers
// FP32 deltas only, and a rounding error is relative to the distance from the anchor rather
// than to the iterate itself: as the restarts close in on the optimum the FP32 iterate keeps
// its accuracy, where a plain FP32 iterate stalls at a few hundred units of FP32 rounding.
template <class T>
constexpr bool kDelta = sizeof(T) == 4;

// dx' = proj_[dl,du](dx - tau (cg + A'dy)): the primal step of pdhg.cpp:392-400 in deltas.
template <class T>
struct PrimalStepDelta {
  const T* x;
  T* xn;
  const double* cg;
  const float* dl;
  const float* du;
  double* xsum;
  double tau;
  int pending;
  struct In {
    double xo, c, lo, hi, xs;
  };
  __device__ __forceinline__ In load(int j) const {
    In v;
    v.xo = ld(x + j);
    v.c = ro(cg + j);
    v.lo = ro(dl + j);
    v.hi = ro(du + j);
    v.xs = pending ? __ldcg(xsum + j) : 0.0;
    return v;
  }
  __device__ __forceinline__ void apply(int j, const double (&s)[1], const In& v,
                                        double (&acc)[3]) const {
    if (pending) xsum[j] = v.xs + v.xo;
    const double xnew = project(v.xo - tau * (v.c + s[0]), v.lo, v.hi);
    const T xs = static_cast<T>(xnew);
    xn[j] = xs;
    const double d = static_cast<double>(xs) - v.xo;
    acc[0] += d * d;
  }
};

// The dual step of pdhg.cpp:402-408 in deltas: with a' = A dx' (this phase), a = A dx,
// A xbar = axr + 2 a' - a and v = yr + dy + sigma A xbar in FP64; dy' = y' - yr.
template <class T>
struct DualStepDelta {
  const T* y;
  T* yn;
  const double* ax;
  double* axn;
  const double* yr;
  const double* axr;
  const double* rl;
  const double* ru;
  double* ysum;
  double sigma;
  int pending;
  struct In {
    double yo, aold, yr, axr, lo, hi, ys;
  };
  __device__ __forceinline__ In load(int i) const {
    In v;
    v.yo = ld(y + i);
    v.aold = __ldcg(ax + i);
    v.yr = ro(yr + i);
    v.axr = ro(axr + i);
    v.lo = ro(rl + i);
    v.hi = ro(ru + i);
    v.ys = pending ? __ldcg(ysum + i) : 0.0;
    return v;
  }
  __device__ __forceinline__ void apply(int i, const double (&s)[1], const In& v,
                                        double (&acc)[3]) const {
    if (pending) ysum[i] = v.ys + v.yo;
    const double anew = s[0];
    const double w = (v.yr + v.yo) + sigma * (v.axr + 2.0 * anew - v.aold);
    const double ynew = w - sigma * project(w / sigma, v.lo, v.hi);
    const T ys = static_cast<T>(ynew - v.yr);
    yn[i] = ys;
    axn[i] = anew;
    const double d = static_cast<double>(ys) - v.yo;
    acc[1] += d * d;
    acc[2] += d * (anew - v.aold);
  }
};

// Column side of the anchor terms: cg = c + A'yr and the bounds relative to xr (an absent
// bound stays absent).
struct AnchorCol {
  const double* c;
  const double* cl;
  const double* cu;
  const double* xr;
  double* cg;
  float* dl;
  float* du;
  struct In {
    double c, lo, hi, xr;
  };
  __device__ __forceinline__ In load(int j) const {
    return In{__ldg(c + j), __ldg(cl + j), __ldg(cu + j), __ldcg(xr + j)};
  }
  __device__ __forceinline__ void apply(int j, const double (&s)[1], const In& v,
                                        double (&)[1]) const {
    cg[j] = v.c + s[0];
    dl[j] = finite_bound(v.lo) ? static_cast<float>(v.lo - v.xr) : -INFINITY;
    du[j] = finite_bound(v.hi) ? static_cast<float>(v.hi - v.xr) : INFINITY;
  }
};

// ---- the Halpern operator ------------------------------------------------------------------
//
// Reflected Halpern PDHG: with T one PDHG step (pdhg.cpp:392-408 at a constant step size),
// z_{k+1} = w (2 T(z_k) - z_k) + (1 - w) z_0, w = (k+1)/(k+2), k the steps since the last
// restart and z_0 the restart point. Phase P forms x' = T(z_k)_x and x_{k+1}; phase D gathers
// x_{k+1}, so a_{k+1} = A x_{k+1} is exact for the stored iterate as in the reference mode,
// and recovers A xbar = A (2x' - x_k) = (a_{k+1} - (1 - w) A x_0) / w for the dual step. On the
// FP32 level everything is a delta from the restart point, where x_0 and A x_0 are zero.

template <class T>
struct PrimalStepHalpern {
  const T* x;
  T* xn;
  T* xt;
  const T* c;
  const T* cl;
  const T* cu;
  const double* x0;
  double tau, w;
  struct In {
    double xo, c, lo, hi, x0;
  };
  __device__ __forceinline__ In load(int j) const {
    return In{ld(x + j), ro(c + j), ro(cl + j), ro(cu + j), __ldcg(x0 + j)};
  }
  __device__ __forceinline__ void apply(int j, const double (&s)[1], const In& v,
                                        double (&)[3]) const {
    const T xp = static_cast<T>(project(v.xo - tau * (v.c + s[0]), v.lo, v.hi));
    xt[j] = xp;
    xn[j] = static_cast<T>(w * (2.0 * static_cast<double>(xp) - v.xo) + (1.0 - w) * v.x0);
  }
};

template <class T>
struct PrimalStepHalpernDelta {
  const T* x;
  T* xn;
  T* xt;
  const double* cg;
  const float* dl;
  const float* du;
  double tau, w;
  struct In {
    double xo, c, lo, hi;
  };
  __device__ __forceinline__ In load(int j) const {
    return In{ld(x + j), ro(cg + j), ro(dl + j), ro(du + j)};
  }
  __device__ __forceinline__ void apply(int j, const double (&s)[1], const In& v,
                                        double (&)[3]) const {
    const T xp = static_cast<T>(project(v.xo - tau * (v.c + s[0]), v.lo, v.hi));
    xt[j] = xp;
    xn[j] = static_cast<T>(w * (2.0 * static_cast<double>(xp) - v.xo));
  }
};

template <class T>
struct DualStepHalpern {
  const T* y;
  T* yn;
  T* yt;
  double* axn;
  const T* rl;
  const T* ru;
  const double* y0;
  const double* ax0;
  double sigma, w;
  struct In {
    double yo, lo, hi, y0, a0;
  };
  __device__ __forceinline__ In load(int i) const {
    return In{ld(y + i), ro(rl + i), ro(ru + i), __ldcg(y0 + i), __ldcg(ax0 + i)};
  }
  __device__ __forceinline__ void apply(int i, const double (&s)[1], const In& v,
                                        double (&)[3]) const {
    const double anew = s[0];
    const double axbar = (anew - (1.0 - w) * v.a0) / w;
    const double u = v.yo + sigma * axbar;
    const T yp = static_cast<T>(u - sigma * project(u / sigma, v.lo, v.hi));
    yt[i] = yp;
    yn[i] = static_cast<T>(w * (2.0 * static_cast<double>(yp) - v.yo) + (1.0 - w) * v.y0);
    axn[i] = anew;
  }
};

template <class T>
struct DualStepHalpernDelta {
  const T* y;
  T* yn;
  T* yt;
  double* axn;
  const double* yr;
  const double* axr;
  const double* rl;
  const double* ru;
  double sigma, w;
  struct In {
    double yo, yr, axr, lo, hi;
  };
  __device__ __forceinline__ In load(int i) const {
    return In{ld(y + i), ro(yr + i), ro(axr + i), ro(rl + i), ro(ru + i)};
  }
  __device__ __forceinline__ void apply(int i, const double (&s)[1], const In& v,
                                        double (&)[3]) const {
    const double anew = s[0];
    const double u = (v.yr + v.yo) + sigma * (v.axr + anew / w);
    const double yp = u - sigma * project(u / sigma, v.lo, v.hi);
    const T dyp = static_cast<T>(yp - v.yr);
    yt[i] = dyp;
    yn[i] = static_cast<T>(w * (2.0 * static_cast<double>(dyp) - v.yo));
    axn[i] = anew;
  }
};

// One Halpern step is always taken: no acceptance test, no step-size change (the constant
// step 0.998 / ||A||_2 keeps tau sigma ||A||^2 < 1); an evaluation every 40 steps.
__device__ __forceinline__ void halpern_control(Ctrl& c) {
  c.cur ^= 1;
  ++c.averaged;  // k, the steps since the last restart
  ++c.iteration;
  ++c.attempts;
  c.pending = 0;
  if (c.iteration % 40 == 0) c.state = kNeedEval;
}

// ---- infeasibility and unboundedness certificates ------------------------------------------
//
// At an evaluation the iterate differences are tested as certificates in the sense of
// src/core/certificate.cpp (the reference's own checkers; its CPU PDHG never produces one):
//
//  * Farkas (primal infeasibility, certificate.cpp:29-119): f = -Dr (y - y_r), the dual
//    movement since the last restart in original units and the reference's row_dual sign.
//    Rows aggregate to S = sum_i f_i * (row_lower if f_i > 0, row_upper if f_i < 0); the
//    column box allows at most M = max over the box of d.x with d = A'f. S > M proves the LP
//    infeasible. For a feasible LP S <= M for every f, so the test cannot fire on one.
//  * primal ray (dual infeasibility, certificate.cpp:121-218): r = Dc (x_k - x_{k-1}), the
//    last accepted step in original units. It must move no column against a finite bound,
//    keep A r off every finite row bound it would cross, and improve the min-space cost.
//
// The device test is a filter with the reference's structure (with a margin for the Farkas
// test, and loose enough for a near-ray that the host can repair); the host re-checks every
// candidate exactly with the reference's rules before it reports one.

// Slots of the row/column terms gathered in the evaluation's first pass. Max-reduced: 1-4, 6.
//   0 S, 1 max|f|, 2 max|f| leaning on a missing row bound,
//   3 max|r|, 4 max|r| against a finite column bound, 5 c'r (min space), 6 max|c_j r_j|
constexpr int kCertSlots = 7;
constexpr unsigned kCertMaxMask = (1u << 1) | (1u << 2) | (1u << 3) | (1u << 4) | (1u << 6);

__device__ __forceinline__ void farkas_row_terms(double f, double lo, double hi,
                                                 double (&e)[kCertSlots]) {
  e[1] = dmax(e[1], fabs(f));
  if (f > 0.0) {
    if (finite_bound(lo)) e[0] += f * lo; else e[2] = dmax(e[2], f);
  } else if (f < 0.0) {
    if (finite_bound(hi)) e[0] += f * hi; else e[2] = dmax(e[2], -f);
  }
}

__device__ __forceinline__ void ray_col_terms(double r, double lo, double hi, double c,
                                              double (&e)[kCertSlots]) {
  e[3] = dmax(e[3], fabs(r));
  if (r > 0.0 && finite_bound(hi)) e[4] = dmax(e[4], r);
  if (r < 0.0 && finite_bound(lo)) e[4] = dmax(e[4], -r);
  e[5] += c * r;
  e[6] = dmax(e[6], fabs(c * r));
}

// sum_k M_ik (u - v)_k: a matrix times the difference of two vectors
template <class U, class V>
struct DiffGather {
  const U* u;
  const V* v;
  __device__ __forceinline__ void add(double (&s)[1], double a, int k) const {
    s[0] += a * (ld(u + k) - ld(v + k));
  }
  __device__ __forceinline__ double product(int, double a, int k) const {
    return a * (ld(u + k) - ld(v + k));
  }
};

// Column terms of the Farkas test for d = A'f = -(A'_scaled (y - y_r)) / Dc.
// slots: 0 max |d|, 1 reachable M, 2 max |d| over columns leaning on a missing bound
constexpr unsigned kFarkasColMaxMask = (1u << 0) | (1u << 2);
struct FarkasCol {
  const double* dc;
  const double* cl0;
  const double* cu0;
  struct In {
    double dc, lo, hi;
  };
  __device__ __forceinline__ In load(int j) const {
    return In{__ldg(dc + j), __ldg(cl0 + j), __ldg(cu0 + j)};
  }
  __device__ __forceinline__ void apply(int j, const double (&s)[1], const In& v,
                                        double (&acc)[3]) const {
    const double d = -s[0] / v.dc;
    acc[0] = dmax(acc[0], fabs(d));
    if (d > 0.0) {
      if (finite_bound(v.hi)) acc[1] += d * v.hi; else acc[2] = dmax(acc[2], d);
    } else if (d < 0.0) {
      if (finite_bound(v.lo)) acc[1] += d * v.lo; else acc[2] = dmax(acc[2], -d);
    }
  }
};

// Row terms of the ray test for A r = (A_scaled (x_k - x_{k-1})) / Dr.
// slots: 0 max |(A r)_i| against a finite row bound, 1 max |(A r)_i|
struct RayRow {
  const double* dr;
  const double* rl0;
  const double* ru0;
  struct In {
    double dr, lo, hi;
  };
  __device__ __forceinline__ In load(int i) const {
    return In{__ldg(dr + i), __ldg(rl0 + i), __ldg(ru0 + i)};
  }
  __device__ __forceinline__ void apply(int i, const double (&s)[1], const In& v,
                                        double (&acc)[2]) const {
    const double act = s[0] / v.dr;
    if (act > 0.0 && finite_bound(v.hi)) acc[0] = dmax(acc[0], act);
    if (act < 0.0 && finite_bound(v.lo)) acc[0] = dmax(acc[0], -act);
    acc[1] = dmax(acc[1], fabs(act));
  }
};

// The device filter: 1 = Farkas candidate, 2 = ray candidate, 0 = neither. Sets
// c.farkas_margin to the normalised Farkas margin S - M when that test ran.
__device__ __forceinline__ int certificate_test(Ctrl& c, const double (&e)[kCertSlots],
                                                const double (&fk)[3], const double (&rr)[2]) {
  if (e[1] > 0.0) {
    const double Sn = e[0] / e[1], Mn = fk[1] / e[1];
    const double margin = Sn - Mn;
    c.farkas_margin = margin;
    const bool rows_ok = e[2] <= 1e-9 * e[1];
    const bool cols_ok = fk[2] <= 1e-9 * dmax(fk[0], 1e-300);
    if (rows_ok && cols_ok && margin > 1e-6 * dmax(1.0, dmax(fabs(Sn), fabs(Mn)))) return 1;
  }
  if (e[3] > 0.0) {
    // looser than the checker: the host repairs a near-ray before its exact check
    const double improvement = e[5] / e[3];
    const bool cols_ok = e[4] <= 1e-3 * e[3];
    const bool rows_ok = rr[0] <= 1e-3 * dmax(e[3], rr[1]);
    if (cols_ok && rows_ok && improvement < -1e-6 * dmax(1.0, e[6] / e[3])) return 2;
  }
  return 0;
}

// The slot of the previous accepted iterate at an evaluation: an evaluation follows an
// accepted step (pdhg.cpp:502-503), which flipped `cur`.
__device__ __forceinline__ int cur_prev_slot(const Ctrl& c) { return c.cur ^ 1; }

// Evaluations between two certificate tests, and after a candidate the host turned down.
constexpr int kCertEvery = 4;
constexpr int kCertCooldown = 8;

// Sum (or max) of kPartSlots-wide block partials over all blocks, in block order. Every
// block calls it after a barrier and gets identical totals.
template <int NS, unsigned MAXMASK>
__device__ __forceinline__ void reduce_partials(const double* partials, int first_slot,
                                                double (&tot)[NS], double* sh) {
  const int G = gridDim.x;
#pragma unroll
  for (int s = 0; s < NS; ++s) tot[s] = 0.0;
  for (int b = threadIdx.x; b < G; b += kThreads) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double v = __ldcg(partials + (size_t)b * kPartSlots + first_slot + s);
      tot[s] = ((MAXMASK >> s) & 1u) ? dmax(tot[s], v) : tot[s] + v;
    }
  }
  block_reduce<NS, MAXMASK>(tot, sh);
}

__device__ __forceinline__ void write_partials(double* partials, int first_slot, const double* v,
                                               int ns) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < ns; ++s) partials[(size_t)blockIdx.x * kPartSlots + first_slot + s] = v[s];
  }
}

__device__ __forceinline__ double* warp_stream() {
  extern __shared__ double dyn_smem[];
  return dyn_smem + (size_t)(threadIdx.x >> 5) * kItemNnz;
}


// Adaptive step size and acceptance (pdhg.cpp:413-496) from the attempt's reductions
// tot = {sum (x'-x)^2, sum (y'-y)^2, sum (y'-y)(A dx)}; flags an evaluation when one is due
// (pdhg.cpp:502-503). One thread calls it.
__device__ __forceinline__ void step_control(Ctrl& c, const double (&tot)[3]) {
  const double movement = 0.5 * c.omega * tot[0] + 0.5 * tot[1] / c.omega;
  const double interaction = fabs(tot[2]);
  const bool no_information = interaction <= 0.0;
  const double limit = no_information ? INFINITY : movement / interaction;
  const double exponent = (double)(c.iteration + 1 > 2 ? c.iteration + 1 : 2);
  const double shrink = 1.0 - pow(exponent, -0.3);
  const double grow = 1.0 + pow(exponent, -0.6);
  const double proposed = dmin(shrink * limit, grow * c.eta);
  const bool accept = c.eta <= limit;
  if (accept) {
    c.cur ^= 1;
    ++c.averaged;
    ++c.iteration;
  }
  c.pending = accept ? 1 : 0;
  if (!no_information) {
    c.eta = proposed < 1e-12 ? 1e-12 : (c.eta_ceiling < proposed ? c.eta_ceiling : proposed);
  }
  ++c.attempts;
  if (c.iteration != 0 && (c.iteration % 40 == 0 || no_information)) c.state = kNeedEval;
}

// ---- the iteration kernel ---------------------------------------------------------------

#ifdef SIH26_PHASE_TIMING
// Instrumented builds only: per-block nanoseconds spent in phase P, barrier 1, phase D,
// barrier 2 and the control step, summed over attempts (read back with
// sih26_phase_timing_read).
__device__ unsigned long long g_phase_ns[4096 * 5];
#define SIH26_MARK(k)                                                  \
  do {                                                                 \
    __syncthreads();                                                   \
    if (threadIdx.x == 0) {                                            \
      const unsigned long long now_ = global_ns();                     \
      g_phase_ns[blockIdx.x * 5 + (k)] += now_ - mark_ns;              \
      mark_ns = now_;                                                  \
    }                                                                  \
  } while (0)
#define SIH26_MARK_START() (mark_ns = threadIdx.x == 0 ? global_ns() : 0ull)
#else
#define SIH26_MARK(k) \
  do {                \
  } while (0)
#define SIH26_MARK_START() (mark_ns = 0ull)
#endif

// One instance per operator (kHalpern: the Halpern operator, else the reference's adaptive
// step), so each carries only its own step's registers.
template <class T, bool kHalpern>
__global__ void __launch_bounds__(kThreads, 2) iterate_kernel(Prob<T> P, State<T> S,
                                                              long long max_attempts) {
  unsigned long long mark_ns = 0;
  (void)mark_ns;
  __shared__ Ctrl c;
  __shared__ double sh[kWarps * 4];
  double* stream = warp_stream();
  if (threadIdx.x == 0) {
    c = *S.ctrl;
    // The deadline flag is read once per launch: the last arriver of a barrier sets it after
    // the barrier opens, so only a read made before this launch's first barrier is the same
    // in every block.
    c.time_up |= *((volatile int*)S.bar.time_up);
  }
  __syncthreads();
  if (c.state != kRunning) return;
  const int G = gridDim.x;
  long long a = 0;
  for (;;) {
    // loop top (pdhg.cpp:384-385)
    if (c.iteration >= c.iteration_limit) {
      if (threadIdx.x == 0) c.state = kIterationLimit;
      break;
    }
    if (c.time_up) {
      if (threadIdx.x == 0) c.state = kTimeLimit;
      break;
    }
    if (a >= max_attempts) break;
    ++a;
    const int cur = c.cur, nxt = cur ^ 1;
    const double tau = c.eta / c.omega;
    const double sigma = c.eta * c.omega;
    double* part = S.partials + (size_t)(c.attempts & 1) * G * kPartSlots;
    double acc[3] = {0.0, 0.0, 0.0};
    SIH26_MARK_START();
    if constexpr (kHalpern) {
      const double w = (double)(c.averaged + 1) / (double)(c.averaged + 2);
      if constexpr (kDelta<T>) {
        PrimalStepHalpernDelta<T> ps{S.x[cur], S.x[nxt], S.xt, S.cg, S.dl, S.du, tau, w};
        run_phase<1, 3, true, true>(P.AT.ptr, P.AT.idx, P.AT.val, P.pati, Gather1<T>{S.y[cur]}, ps, acc, stream);
      } else {
        PrimalStepHalpern<T> ps{S.x[cur], S.x[nxt], S.xt, P.c, P.cl, P.cu, S.xr, tau, w};
        run_phase<1, 3, true, true>(P.AT.ptr, P.AT.idx, P.AT.val, P.pati, Gather1<T>{S.y[cur]}, ps, acc, stream);
      }
      SIH26_MARK(0);
      if (!grid_barrier(S.bar)) goto device_error;
      SIH26_MARK(1);
      if constexpr (kDelta<T>) {
        DualStepHalpernDelta<T> ds{S.y[cur], S.y[nxt], S.yt, S.ax[nxt], S.yr, S.axr, P.rl64,
                                   P.ru64, sigma, w};
        run_phase<1, 3, true, true>(P.A.ptr, P.A.idx, P.A.val, P.pai, Gather1<T>{S.x[nxt]}, ds, acc, stream);
      } else {
        DualStepHalpern<T> ds{S.y[cur], S.y[nxt], S.yt, S.ax[nxt], P.rl, P.ru, S.yr, S.axr, sigma, w};
        run_phase<1, 3, true, true>(P.A.ptr, P.A.idx, P.A.val, P.pai, Gather1<T>{S.x[nxt]}, ds, acc, stream);
      }
      SIH26_MARK(2);
      if (!grid_barrier(S.bar)) goto device_error;
      SIH26_MARK(3);
      if (threadIdx.x == 0) halpern_control(c);
      __syncthreads();
      SIH26_MARK(4);
      if (c.state != kRunning) break;
      continue;
    }
    if constexpr (kDelta<T>) {
      PrimalStepDelta<T> ps{S.x[cur], S.x[nxt], S.cg, S.dl, S.du, S.xsum, tau, c.pending};
      run_phase<1, 3, false, true>(P.AT.ptr, P.AT.idx, P.AT.val, P.pati, Gather1<T>{S.y[cur]}, ps, acc, stream);
    } else {
      PrimalStep<T> ps{S.x[cur], S.x[nxt], P.c, P.cl, P.cu, S.xsum, tau, c.pending};
      run_phase<1, 3, false, true>(P.AT.ptr, P.AT.idx, P.AT.val, P.pati, Gather1<T>{S.y[cur]}, ps, acc, stream);
    }
    SIH26_MARK(0);
    if (!grid_barrier(S.bar)) goto device_error;
    SIH26_MARK(1);

    if constexpr (kDelta<T>) {
      DualStepDelta<T> ds{S.y[cur], S.y[nxt], S.ax[cur], S.ax[nxt], S.yr, S.axr, P.rl64,
                          P.ru64, S.ysum, sigma, c.pending};
      run_phase<1, 3, false, true>(P.A.ptr, P.A.idx, P.A.val, P.pai, Gather1<T>{S.x[nxt]}, ds, acc, stream);
    } else {
      DualStep<T> ds{S.y[cur], S.y[nxt], S.ax[cur], S.ax[nxt], P.rl, P.ru, S.ysum, sigma, c.pending};
      run_phase<1, 3, false, true>(P.A.ptr, P.A.idx, P.A.val, P.pai, Gather1<T>{S.x[nxt]}, ds, acc, stream);
    }
    SIH26_MARK(2);
    block_reduce<3, 0u>(acc, sh);
    write_partials(part, 0, acc, 3);
    if (!grid_barrier(S.bar)) goto device_error;
    SIH26_MARK(3);

    {
      double tot[3];
      reduce_partials<3, 0u>(part, 0, tot, sh);
      if (threadIdx.x == 0) step_control(c, tot);
      __syncthreads();
      SIH26_MARK(4);
      if (c.state != kRunning) break;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *S.ctrl = c;
  return;
device_error:
  if (blockIdx.x == 0 && threadIdx.x == 0) S.ctrl->state = kDeviceError;
}

// A x for the starting point, through the same phase code and partition as phase D, so that
// A x' - A x is exactly zero whenever x' == x (the reference's interaction is then exactly
// zero, pdhg.cpp:424-438, 454).
template <class T>
__global__ void __launch_bounds__(kThreads, 2) init_ax_kernel(Prob<T> P, State<T> S) {
  double* stream = warp_stream();
  double dummy[1] = {0.0};
  const int cur = S.ctrl->cur;
  run_phase<1, 1, false, true>(P.A.ptr, P.A.idx, P.A.val, P.pai, Gather1<T>{S.x[cur]},
                               StoreRow<1>{S.ax[cur], -1}, dummy, stream);
}

// out = M v over one partition with nothing fused: the autotuner times candidate schedules
// with it.
template <class T>
__global__ void __launch_bounds__(kThreads, 2) probe_kernel(const int* ptr, const int* idx,
                                                            const T* val, Part part, const T* v,
                                                            double* out) {
  double* stream = warp_stream();
  double dummy[1] = {0.0};
  run_phase<1, 1, false, true>(ptr, idx, val, part, Gather1<T>{v}, StoreRow<1>{out, -1}, dummy,
                               stream);
}

// The slice arrays of a sliced partition from the permuted CSR (one warp per slice item): entry
// k of row row_begin + l at offset + k * rows + l, in the level's value type; padding past a
// row's end holds column 0 and value 0 and is never summed.
template <class T>
__global__ void slice_fill_kernel(const int* __restrict__ ptr, const int* __restrict__ idx,
                                  const double* __restrict__ val, const int4* __restrict__ items,
                                  int count, int* __restrict__ sidx, T* __restrict__ sval) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < count; it += warps) {
    const int4 item = items[it];
    if (item.z >= 0) continue;
    const int rows = item.y - item.x, L = -item.z;
    if (lane >= rows) continue;
    const int r = item.x + lane, b = ptr[r], len = ptr[r + 1] - b;
    for (int k = 0; k < L; ++k) {
      const size_t o = (size_t)item.w + (size_t)k * rows + lane;
      sidx[o] = k < len ? idx[b + k] : 0;
      sval[o] = k < len ? static_cast<T>(val[b + k]) : T(0);
    }
  }
}

// The FP32 level's anchor terms from (xr, yr), FP64 values: axr = A xr, cg = c + A'yr, the
// relative bounds. Needs xr and yr complete in every block.
template <class T>
__device__ __forceinline__ void anchor_phases(const Prob<T>& P, const State<T>& S,
                                              double* stream) {
  double dummy[1] = {0.0};
  run_phase<1, 1>(P.A.ptr, P.A.idx, P.A.val64, P.pa, Gather1<double>{S.xr},
                  StoreRow<1>{S.axr, -1}, dummy, stream);
  run_phase<1, 1>(P.AT.ptr, P.AT.idx, P.AT.val64, P.pat, Gather1<double>{S.yr},
                  AnchorCol{P.c64, P.cl64, P.cu64, S.xr, S.cg, S.dl, S.du}, dummy, stream);
}

// Start of the FP32 level: the anchor terms of the starting anchor (the deltas start at 0).
template <class T>
__global__ void __launch_bounds__(kThreads, 2) anchor_kernel(Prob<T> P, State<T> S) {
  double* stream = warp_stream();
  anchor_phases(P, S, stream);
}

// ---- evaluation ---------------------------------------------------------------------------

// Row terms of evaluate() (pdhg.cpp:152-170, 205-222, 227-238) for NC candidates.
// slots: 0/1 primal violation^2, 2/3 support, 4/5 row dual violation^2, 6/7 complementarity.
template <class T, int NC>
struct RowEval {
  const double* dr;
  const double* rl0;
  const double* ru0;
  const T* y;          // candidate 0 (scaled)
  const double* yavg;  // candidate 1 (scaled)
  const double* ycand; // when non-null: candidate 0 in FP64 (the report)
  double* y_out;       // report: unscaled multipliers
  const double2* pair; // when non-null: both candidates side by side (State::yc)
  struct In {
    double dr, lo, hi, y0, y1;
  };
  __device__ __forceinline__ In load(int i) const {
    In v;
    v.dr = __ldg(dr + i);
    v.lo = __ldg(rl0 + i);
    v.hi = __ldg(ru0 + i);
    if (pair) {
      const double2 t = __ldcg(pair + i);
      v.y0 = t.x;
      v.y1 = t.y;
    } else {
      v.y0 = ycand ? __ldcg(ycand + i) : ld(y + i);
      v.y1 = NC > 1 ? __ldcg(yavg + i) : 0.0;
    }
    return v;
  }
  // acc holds slots 0 .. NS-1 (the row pass of the evaluation keeps only its own 8)
  template <int NS>
  __device__ __forceinline__ void apply(int i, const double (&s)[NC], const In& v,
                                        double (&acc)[NS]) const {
    static_assert(NS >= 8, "the row terms fill slots 0-7");
    const double lo = v.lo, hi = v.hi;
#pragma unroll
    for (int q = 0; q < NC; ++q) {
      const double act = s[q] / v.dr;
      const double yi = (q == 0 ? v.y0 : v.y1) * v.dr;
      if (y_out && q == 0) y_out[i] = yi;
      double viol = 0.0;
      if (finite_bound(lo)) viol = dmax(viol, lo - act);
      if (finite_bound(hi)) viol = dmax(viol, act - hi);
      acc[0 + q] += viol * viol;
      if (y_out && q == 0) acc[1] = dmax(acc[1], viol);  // report: largest row violation
      if (yi > 0.0) {
        if (finite_bound(hi)) acc[2 + q] += yi * hi; else acc[4 + q] += yi * yi;
      } else if (yi < 0.0) {
        if (finite_bound(lo)) acc[2 + q] += yi * lo; else acc[4 + q] += yi * yi;
      }
      if (lo != hi) {
        const double ls = finite_bound(lo) ? act - lo : INFINITY;
        const double us = finite_bound(hi) ? hi - act : INFINITY;
        acc[6 + q] = dmax(acc[6 + q], fabs(yi) * dmin(ls, us));
      }
    }
  }
};

// Column terms (pdhg.cpp:172-199, 239-256). slots: 8/9 dual violation^2, 10/11 bound
// contribution, 12/13 complementarity, 14/15 primal objective. The report variant also
// writes the unscaled point and reduced costs. acc[0] is slot kBase: the column pass of the
// evaluation keeps only slots 8-15 (kBase 8), the others the whole 16.
template <class T, int NC, int kBase = 0>
struct ColEval {
  const double* dc;
  const double* cl0;
  const double* cu0;
  const double* c0;
  const T* x;
  const double* xavg;
  const double* xcand;  // report: candidate 0 in FP64
  double* x_out;        // report outputs (unscaled, permuted order)
  double* reduced_out;
  const double2* pair;  // when non-null: both candidates side by side (State::xc)
  struct In {
    double dc, lo, hi, c, x0, x1;
  };
  __device__ __forceinline__ In load(int j) const {
    In v;
    v.dc = __ldg(dc + j);
    v.lo = __ldg(cl0 + j);
    v.hi = __ldg(cu0 + j);
    v.c = __ldg(c0 + j);
    if (pair) {
      const double2 t = __ldcg(pair + j);
      v.x0 = t.x;
      v.x1 = t.y;
    } else {
      v.x0 = xcand ? __ldcg(xcand + j) : ld(x + j);
      v.x1 = NC > 1 ? __ldcg(xavg + j) : 0.0;
    }
    return v;
  }
  template <int NS>
  __device__ __forceinline__ void apply(int j, const double (&s)[NC], const In& v,
                                        double (&acc)[NS]) const {
    static_assert(kBase + NS >= 16 && kBase <= 8, "the column terms fill slots 8-15");
    const double lo = v.lo, hi = v.hi;
#pragma unroll
    for (int q = 0; q < NC; ++q) {
      const double d = v.c + s[q] / v.dc;
      const double xj = (q == 0 ? v.x0 : v.x1) * v.dc;
      if (x_out && q == 0) {
        x_out[j] = xj;
        reduced_out[j] = d;
        // report: largest column bound violation
        if (finite_bound(lo)) acc[9 - kBase] = dmax(acc[9 - kBase], lo - xj);
        if (finite_bound(hi)) acc[9 - kBase] = dmax(acc[9 - kBase], xj - hi);
      }
      if (d > 0.0) {
        if (finite_bound(lo)) acc[10 + q - kBase] += d * lo; else acc[8 + q - kBase] += d * d;
      } else if (d < 0.0) {
        if (finite_bound(hi)) acc[10 + q - kBase] += d * hi; else acc[8 + q - kBase] += d * d;
      }
      if (lo != hi) {
        const double ls = finite_bound(lo) ? xj - lo : INFINITY;
        const double us = finite_bound(hi) ? hi - xj : INFINITY;
        acc[12 + q - kBase] = dmax(acc[12 + q - kBase], fabs(d) * dmin(ls, us));
      }
      acc[14 + q - kBase] += v.c * xj;
    }
  }
};

__device__ __forceinline__ Residuals make_residuals(const double* t, int q, double bound_norm,
                                                    double cost_norm) {
  Residuals r;
  r.absolute_primal = sqrt(t[0 + q]);
  r.primal = r.absolute_primal / (1.0 + bound_norm);
  r.absolute_dual = sqrt(t[8 + q] + t[4 + q]);
  r.dual = r.absolute_dual / (1.0 + cost_norm);
  r.complementarity = dmax(t[6 + q], t[12 + q]);
  r.primal_objective = t[14 + q];
  r.dual_objective = t[10 + q] - t[2 + q];
  const double absolute_gap = fabs(r.primal_objective - r.dual_objective);
  r.gap = absolute_gap / (1.0 + fabs(r.primal_objective) + fabs(r.dual_objective));
  r.gap_as_verified = absolute_gap / dmax(1.0, fabs(r.primal_objective));
  return r;
}

__device__ __forceinline__ double worst(const Residuals& r) { return dmax(dmax(r.primal, r.dual), r.gap); }

// pdhg.cpp:119-131
__device__ __forceinline__ bool meets_request(const Residuals& r, double tol) {
  return r.primal <= tol && r.dual <= tol && r.gap <= tol && r.absolute_primal <= 1e-7;
}
__device__ __forceinline__ bool meets_project_standard(const Residuals& r) {
  return r.absolute_primal <= 1e-7 && r.absolute_dual <= 1e-7 && r.gap_as_verified <= 1e-9 &&
         r.complementarity <= 1e-6;
}


// The evaluation's decisions (pdhg.cpp:505-643) from the reduced residual terms t (slots of
// RowEval / ColEval) and the movement since the last restart mv = {|x-x_r|^2, |y-y_r|^2}:
// candidate choice, best point, stopping test, restart and primal weight. Sets
// flags = {best updated, restart, chosen is the average}. One thread calls it.
__device__ __forceinline__ void evaluation_decision(Ctrl& c, const double (&t)[kEvalSlots],
                                                    const double (&mv)[2], bool has_average,
                                                    int* flags) {
  ++c.evaluations;
  c.pending = 0;
  const Residuals current = make_residuals(t, 0, c.bound_norm, c.cost_norm);
  Residuals better = current;
  int chosen_average = 0;
  if (has_average) {
    const Residuals average = make_residuals(t, 1, c.bound_norm, c.cost_norm);
    c.average = average;
    if (worst(average) < worst(current)) {
      better = average;
      chosen_average = 1;
    }
  }
  c.current = current;
  c.chosen_average = chosen_average;
  int best_updated = 0, restart = 0;
  if (worst(better) < c.best_worst) {
    c.best = better;
    c.best_worst = worst(better);
    best_updated = 1;
  }
  bool stop_here;
  if (c.stop_rule == 1) {
    stop_here = worst(better) <= c.tolerance;
  } else {
    stop_here = meets_request(better, c.tolerance) &&
                (c.stop_at_request || meets_project_standard(better));
  }
  if (stop_here) {
    c.best = better;
    c.best_worst = worst(better);
    best_updated = 1;
    c.converged = 1;
    c.state = kConverged;
  } else {
    c.state = kRunning;
    if (c.use_restarts) {
      const double kkt = worst(better);
      const long long since = c.iteration - c.last_restart;
      const bool sufficient = kkt <= 0.2 * c.restart_kkt;
      const long long art = (long long)(0.36 * (double)c.iteration);
      const bool artificial = since >= (art > 40 ? art : 40);
      if (sufficient || artificial) {
        const double dx_norm = sqrt(mv[0]), dy_norm = sqrt(mv[1]);
        if (dx_norm > 1e-12 && dy_norm > 1e-12) {
          const double theta = 0.5;
          double w = exp(theta * log(dy_norm / dx_norm) + (1.0 - theta) * log(c.omega));
          c.omega = w < 1e-6 ? 1e-6 : (1e6 < w ? 1e6 : w);
        }
        c.averaged = 0;
        c.restart_kkt = kkt;
        c.last_restart = c.iteration;
        ++c.restarts;
        restart = 1;
      }
    }
  }
  c.best_is_set |= best_updated;
  flags[0] = best_updated;
  flags[1] = restart;
  flags[2] = chosen_average;
}

template <class T>
__global__ void __launch_bounds__(kThreads, 2) evaluate_kernel(Prob<T> P, State<T> S) {
  __shared__ Ctrl c;
  __shared__ double sh[kWarps * kEvalSlots];
  __shared__ int flags[4];  // best updated, restart, chosen average, certificate kind
  double* stream = warp_stream();
  if (threadIdx.x == 0) c = *S.ctrl;
  __syncthreads();
  if (c.state != kNeedEval) return;
  // every kCertEvery-th evaluation tests the iterate differences as certificates
  const bool test_cert = c.farkas_cooldown == 0 && (c.evaluations % kCertEvery) == kCertEvery - 1;
  const int prev = cur_prev_slot(c);
  double cert_scale = 1.0;  // max|f| or max|r| of a candidate, once one is found
  const int G = gridDim.x;
  const int cur = c.cur;
  const int stride = G * kThreads;
  const int gt = blockIdx.x * kThreads + threadIdx.x;
  const bool has_average = c.averaged > 0;
  const double count = (double)c.averaged;
  double* part = S.partials;  // slots 0-1 restart movement, 2-17 residual terms

  // E1: fold the pending running-sum term, form the scaled averages, and measure the
  // movement since the last restart (pdhg.cpp:519-528, 613-624).
  // On the FP32 level the iterates and sums are deltas from the anchor: the movement is the
  // delta itself, and the full FP64 iterate goes to xc / yc (beside the second candidate)
  // for the passes below.
  double acc1[2] = {0.0, 0.0};
  double ec[kCertSlots];
#pragma unroll
  for (int s = 0; s < kCertSlots; ++s) ec[s] = 0.0;
  // the Halpern operator's second candidate is the PDHG output T(z_k), not an average
  const bool halpern = c.halpern != 0;
  const T* ray_from = halpern ? S.xt : S.x[cur];
  for (int j = gt; j < P.n; j += stride) {
    const double xo = ld(S.x[cur] + j);
    const double xs = S.xsum[j] + (c.pending ? xo : 0.0);
    S.xsum[j] = xs;
    double d;
    if constexpr (kDelta<T>) {
      const double r = S.xr[j];
      S.xc[j] = make_double2(r + xo, has_average ? r + (halpern ? ld(S.xt + j) : xs / count) : 0.0);
      d = xo;
    } else {
      S.xc[j] = make_double2(xo, has_average ? (halpern ? ld(S.xt + j) : xs / count) : 0.0);
      d = xo - ld(S.xr + j);
    }
    acc1[0] += d * d;
    if (test_cert) {
      const double r = __ldg(P.dc + j) * (ld(ray_from + j) - ld(S.x[prev] + j));
      ray_col_terms(r, __ldg(P.cl0 + j), __ldg(P.cu0 + j), __ldg(P.c0 + j), ec);
    }
  }
  for (int i = gt; i < P.m; i += stride) {
    const double yo = ld(S.y[cur] + i);
    const double ys = S.ysum[i] + (c.pending ? yo : 0.0);
    S.ysum[i] = ys;
    double d;
    if constexpr (kDelta<T>) {
      const double r = S.yr[i];
      S.yc[i] = make_double2(r + yo, has_average ? r + (halpern ? ld(S.yt + i) : ys / count) : 0.0);
      d = yo;
    } else {
      S.yc[i] = make_double2(yo, has_average ? (halpern ? ld(S.yt + i) : ys / count) : 0.0);
      d = yo - ld(S.yr + i);
    }
    acc1[1] += d * d;
    if (test_cert) farkas_row_terms(-__ldg(P.dr + i) * d, __ldg(P.rl0 + i), __ldg(P.ru0 + i), ec);
  }
  block_reduce<2, 0u>(acc1, sh);
  write_partials(part, 0, acc1, 2);
  if (test_cert) {
    block_reduce<kCertSlots, kCertMaxMask>(ec, sh);
    write_partials(part, 18, ec, kCertSlots);
  }
  if (!grid_barrier(S.bar)) goto device_error;

  {
    // E2: both candidates' residual terms in one pass over each matrix (FP64 values, the
    // FP64 slices): one 16-byte gather per entry reads both candidates.
    // Each pass keeps only its own 8 slots live (rows 0-7, columns 8-15); every slot is
    // reduced on its own, so the split changes no sum. The epilogue's inputs (five or six
    // FP64 values a row) are loaded after the row's sum (kLateIn), which leaves the registers
    // to four paired gathers per round (measured fastest of 2 / 4, early / late).
    {
      double acc[8];
#pragma unroll
      for (int s = 0; s < 8; ++s) acc[s] = 0.0;
      RowEval<T, 2> re{P.dr, P.rl0, P.ru0, nullptr, nullptr, nullptr, nullptr, S.yc};
      run_phase<2, 8, false, true, 4, true>(P.A.ptr, P.A.idx, P.A.val64, P.pae, GatherPair{S.xc},
                                            re, acc, stream);
      block_reduce<8, kEvalMaxMask & 0xffu>(acc, sh);
      write_partials(part, 2, acc, 8);
    }
    {
      double acc[8];
#pragma unroll
      for (int s = 0; s < 8; ++s) acc[s] = 0.0;
      ColEval<T, 2, 8> ce{P.dc, P.cl0, P.cu0, P.c0, nullptr, nullptr, nullptr, nullptr, nullptr,
                          S.xc};
      run_phase<2, 8, false, true, 4, true>(P.AT.ptr, P.AT.idx, P.AT.val64, P.pate,
                                            GatherPair{S.yc}, ce, acc, stream);
      block_reduce<8, (kEvalMaxMask >> 8)>(acc, sh);
      write_partials(part, 10, acc, 8);
    }
    if (test_cert) {
      // the certificates' matrix terms: A'(y - y_r) for the Farkas test, A (x_k - x_{k-1})
      // for the ray test
      double fk[3] = {0.0, 0.0, 0.0};
      if constexpr (kDelta<T>) {
        run_phase<1, 3>(P.AT.ptr, P.AT.idx, P.AT.val64, P.pat, Gather1<T>{S.y[cur]},
                        FarkasCol{P.dc, P.cl0, P.cu0}, fk, stream);
      } else {
        run_phase<1, 3>(P.AT.ptr, P.AT.idx, P.AT.val64, P.pat, DiffGather<T, double>{S.y[cur], S.yr},
                        FarkasCol{P.dc, P.cl0, P.cu0}, fk, stream);
      }
      block_reduce<3, kFarkasColMaxMask>(fk, sh);
      write_partials(part, 25, fk, 3);
      double rr[2] = {0.0, 0.0};
      run_phase<1, 2>(P.A.ptr, P.A.idx, P.A.val64, P.pa, DiffGather<T, T>{ray_from, S.x[prev]},
                      RayRow{P.dr, P.rl0, P.ru0}, rr, stream);
      block_reduce<2, 3u>(rr, sh);
      write_partials(part, 28, rr, 2);
    }
  }
  if (!grid_barrier(S.bar)) goto device_error;

  {
    double mv[2];
    reduce_partials<2, 0u>(part, 0, mv, sh);
    double t[kEvalSlots];
    reduce_partials<kEvalSlots, kEvalMaxMask>(part, 2, t, sh);
    double ect[kCertSlots] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, fkt[3] = {0.0, 0.0, 0.0},
           rrt[2] = {0.0, 0.0};
    if (test_cert) {
      reduce_partials<kCertSlots, kCertMaxMask>(part, 18, ect, sh);
      reduce_partials<3, kFarkasColMaxMask>(part, 25, fkt, sh);
      reduce_partials<2, 3u>(part, 28, rrt, sh);
    }
    if (threadIdx.x == 0) {
      const Ctrl before = c;
      evaluation_decision(c, t, mv, has_average, flags);
      flags[3] = 0;
      if (c.farkas_cooldown > 0) --c.farkas_cooldown;
      if (test_cert && c.state != kConverged) {
        const int kind = certificate_test(c, ect, fkt, rrt);
        if (kind != 0) {
          // keep the restart anchor and the step state as they were: the certificate is read
          // from them, and the loop resumes from them if the host turns it down
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
    if (flags[3] != 0) cert_scale = flags[3] == 1 ? ect[1] : ect[3];
  }
  if (flags[3] == 1) {
    for (int i = gt; i < P.m; i += stride) {
      const double d = kDelta<T> ? ld(S.y[cur] + i) : ld(S.y[cur] + i) - ld(S.yr + i);
      S.cert_row[i] = -__ldg(P.dr + i) * d / cert_scale;
    }
  } else if (flags[3] == 2) {
    for (int j = gt; j < P.n; j += stride)
      S.cert_col[j] = __ldg(P.dc + j) * (ld(ray_from + j) - ld(S.x[prev] + j)) / cert_scale;
  }

  // E3: keep the best point (scaled, FP64) and reset the average at a restart.
  if (flags[0] || flags[1]) {
    for (int j = gt; j < P.n; j += stride) {
      const double2 xcj = S.xc[j];
      const double xo = xcj.x;
      if (flags[0]) S.best_x[j] = flags[2] ? xcj.y : xo;
      if (flags[1]) {
        S.xr[j] = xo;
        S.xsum[j] = 0.0;
        if constexpr (kDelta<T>) S.x[cur][j] = T(0);
      }
    }
    for (int i = gt; i < P.m; i += stride) {
      const double2 yci = S.yc[i];
      const double yo = yci.x;
      if (flags[0]) S.best_y[i] = flags[2] ? yci.y : yo;
      if (flags[1]) {
        S.yr[i] = yo;
        S.ysum[i] = 0.0;
        if constexpr (kDelta<T>) {
          S.y[cur][i] = T(0);
          S.ax[cur][i] = 0.0;
        } else {
          if (halpern) S.axr[i] = S.ax[cur][i];  // A x_0 of the new restart point
        }
      }
    }
  }
  if constexpr (kDelta<T>) {
    // a restart moved the anchor: form its terms (every block takes the same branch)
    if (flags[1]) {
      if (!grid_barrier(S.bar)) goto device_error;
      anchor_phases(P, S, stream);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *S.ctrl = c;
  return;
device_error:
  if (blockIdx.x == 0 && threadIdx.x == 0) S.ctrl->state = kDeviceError;
}

// ---- quality of the reported point ------------------------------------------------------
//
// Solution::recompute_quality (src/core/model.cpp:228-424) on the device, from the reported
// point in original units (x_out, y_out = the PDHG multiplier y, whose reference row_dual is
// -sense y, and red_out = c + A'y in min space, whose sign-folded col_dual is red_out itself)
// and the scaled FP64 point the matrix terms are formed from: a_ij x_j = (A^_ij x^_j) / Dr_i
// and a_ij row_dual_i = -sense (A^_ij y^_i) / Dc_j. One warp per row of A, then per row of
// A' (column of A); `wid` of `wtot` warps. Each term is the reference's term; only the
// rounding of the sums and of the scaled products differs.
__device__ __forceinline__ double nearest_bound_distance(double v, double lo, double hi) {
  double d = INFINITY;
  if (finite_bound(lo)) d = dmin(d, fabs(v - lo));
  if (finite_bound(hi)) d = dmin(d, fabs(v - hi));
  return d;
}

template <class T>
__device__ __forceinline__ void quality_pass(const Prob<T>& P, const double* bx, const double* by,
                                             const double* x_out, const double* y_out,
                                             const double* red_out, int wid, int wtot,
                                             double (&q)[kQualitySlots]) {
  const int lane = threadIdx.x & 31;
  // rows: activity, the row's term scale max(1, max_j |a_ij x_j|), bounds, row prices
  for (int i = wid; i < P.m; i += wtot) {
    double sum = 0.0, big = 0.0;
    const int kb = __ldg(P.A.ptr + i), ke = __ldg(P.A.ptr + i + 1);
    for (int k = kb + lane; k < ke; k += 32) {
      const double t = __ldg(P.A.val64 + k) * __ldcg(bx + __ldg(P.A.idx + k));
      sum += t;
      big = dmax(big, fabs(t));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      sum += __shfl_xor_sync(0xffffffffu, sum, off);
      big = dmax(big, __shfl_xor_sync(0xffffffffu, big, off));
    }
    if (lane == 0) {
      const double dr = __ldg(P.dr + i), lo = __ldg(P.rl0 + i), hi = __ldg(P.ru0 + i);
      const double act = sum / dr;
      const double scale = dmax(1.0, big / dr);
      if (finite_bound(lo) && lo - act > 0.0) {
        q[0] = dmax(q[0], lo - act);
        q[1] = dmax(q[1], (lo - act) / scale);
      }
      if (finite_bound(hi) && act - hi > 0.0) {
        q[0] = dmax(q[0], act - hi);
        q[1] = dmax(q[1], (act - hi) / scale);
      }
      const double yref = -__ldcg(y_out + i);  // sense * row_dual
      q[7] = dmax(q[7], fabs(yref));
      if (lo != hi) {
        double sign = 0.0;
        if (yref > 0.0 && !finite_bound(lo)) sign = yref;
        if (yref < 0.0 && !finite_bound(hi)) sign = -yref;
        if (sign > 0.0) {
          q[2] = dmax(q[2], sign);
          q[5] = dmax(q[5], sign);
        }
        const double slack = nearest_bound_distance(act, lo, hi);
        if (yref != 0.0 && finite_bound(slack)) {
          const double product = fabs(yref) * slack;
          q[4] = dmax(q[4], product);
          q[6] = dmax(q[6], product / scale);
        }
      }
    }
  }
  // columns: bounds, the consistency of col_dual with c - A'row_dual, sign, complementarity
  for (int j = wid; j < P.n; j += wtot) {
    double sum = 0.0, big = 0.0;
    const int kb = __ldg(P.AT.ptr + j), ke = __ldg(P.AT.ptr + j + 1);
    for (int k = kb + lane; k < ke; k += 32) {
      const double t = __ldg(P.AT.val64 + k) * __ldcg(by + __ldg(P.AT.idx + k));
      sum += t;
      big = dmax(big, fabs(t));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      sum += __shfl_xor_sync(0xffffffffu, sum, off);
      big = dmax(big, __shfl_xor_sync(0xffffffffu, big, off));
    }
    if (lane == 0) {
      const double dc = __ldg(P.dc + j), lo = __ldg(P.cl0 + j), hi = __ldg(P.cu0 + j);
      const double c = __ldg(P.c0 + j);
      const double x = __ldcg(x_out + j), d = __ldcg(red_out + j);
      const double xs = dmax(1.0, fabs(x));
      if (finite_bound(lo) && lo - x > 0.0) {
        q[0] = dmax(q[0], lo - x);
        q[1] = dmax(q[1], (lo - x) / xs);
      }
      if (finite_bound(hi) && x - hi > 0.0) {
        q[0] = dmax(q[0], x - hi);
        q[1] = dmax(q[1], (x - hi) / xs);
      }
      const double scale = dmax(1.0, dmax(fabs(c), big / dc));
      const double gap = fabs(c + sum / dc - d);  // |implied - col_dual|, sign folded
      if (gap > 0.0) {
        q[2] = dmax(q[2], gap);
        q[3] = dmax(q[3], gap / scale);
      }
      if (lo != hi) {
        double sign = 0.0;
        if (d > 0.0 && !finite_bound(lo)) sign = d;
        if (d < 0.0 && !finite_bound(hi)) sign = -d;
        if (sign > 0.0) {
          q[2] = dmax(q[2], sign);
          q[3] = dmax(q[3], sign / scale);
        }
        const double slack = nearest_bound_distance(x, lo, hi);
        if (d != 0.0 && finite_bound(slack)) {
          const double product = fabs(d) * slack;
          q[4] = dmax(q[4], product);
          q[3] = dmax(q[3], product / (scale * xs));
        }
      }
    }
  }
}

// Final report (pdhg.cpp:647-661): residuals of the best point, its unscaled value, reduced
// costs and multipliers. Writes the residual block to ctrl->best.
template <class T>
__global__ void __launch_bounds__(kThreads, 2) report_kernel(Prob<T> P, State<T> S, double* x_out,
                                                             double* reduced_out, double* y_out) {
  __shared__ double sh[kWarps * kEvalSlots];
  double* stream = warp_stream();
  double acc[kEvalSlots];
#pragma unroll
  for (int s = 0; s < kEvalSlots; ++s) acc[s] = 0.0;
  RowEval<T, 1> re{P.dr, P.rl0, P.ru0, nullptr, nullptr, S.best_y, y_out};
  run_phase<1, kEvalSlots>(P.A.ptr, P.A.idx, P.A.val64, P.pa, Gather1<double>{S.best_x}, re, acc,
                           stream);
  ColEval<T, 1> ce{P.dc, P.cl0, P.cu0, P.c0, nullptr, nullptr, S.best_x, x_out, reduced_out};
  run_phase<1, kEvalSlots>(P.AT.ptr, P.AT.idx, P.AT.val64, P.pat, Gather1<double>{S.best_y}, ce,
                           acc, stream);
  block_reduce<kEvalSlots, kReportMaxMask>(acc, sh);
  write_partials(S.partials, 2, acc, kEvalSlots);
  if (!grid_barrier(S.bar)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) S.ctrl->state = kDeviceError;
    return;
  }
  double t[kEvalSlots];
  reduce_partials<kEvalSlots, kReportMaxMask>(S.partials, 2, t, sh);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S.ctrl->best = make_residuals(t, 0, S.ctrl->bound_norm, S.ctrl->cost_norm);
    S.ctrl->primal_violation = dmax(0.0, dmax(t[1], t[9]));
  }
  // quality of the reported point, read back after the barrier above
  double qv[kQualitySlots];
#pragma unroll
  for (int k = 0; k < kQualitySlots; ++k) qv[k] = 0.0;
  quality_pass(P, S.best_x, S.best_y, x_out, y_out, reduced_out,
               (int)((blockIdx.x * kThreads + threadIdx.x) >> 5), (int)(gridDim.x * kWarps), qv);
  block_reduce<kQualitySlots, 0xFFu>(qv, sh);
  write_partials(S.partials, 2 + kEvalSlots, qv, kQualitySlots);
  if (!grid_barrier(S.bar)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) S.ctrl->state = kDeviceError;
    return;
  }
  reduce_partials<kQualitySlots, 0xFFu>(S.partials, 2 + kEvalSlots, qv, sh);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < kQualitySlots; ++k) S.ctrl->quality[k] = qv[k];
  }
}

// FP32 -> FP64 hand-over of the mixed-precision mode: the FP32 level's restart state into
// the FP64 level -- iterate (into slot 0), restart anchor and running sums, the deltas added
// back to the anchor (`count` iterates are summed). With `restart` (the Halpern operator) the
// FP64 level restarts at the hand-over point instead: the anchor is the iterate itself.
static __global__ void handover_kernel(State<float> from, int cur, double count, State<double> to,
                                       int m, int n, int restart) {
  const int stride = gridDim.x * blockDim.x;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
    const double r = from.xr[j];
    const double x = r + static_cast<double>(from.x[cur][j]);
    to.x[0][j] = x;
    to.xr[j] = restart ? x : r;
    to.xsum[j] = restart ? 0.0 : count * r + from.xsum[j];
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) {
    const double r = from.yr[i];
    const double y = r + static_cast<double>(from.y[cur][i]);
    to.y[0][i] = y;
    to.yr[i] = restart ? y : r;
    to.ysum[i] = restart ? 0.0 : count * r + from.ysum[i];
  }
}

// ---- norm estimate -----------------------------------------------------------------------

// Power iteration on A'A for ||A||_2 (src/la/scaling.cpp:161-194), cooperative: per step
// normalise v, u = A v, v = A' u, norm = ||v||^(1/2). Writes the estimate (x1.01) to *out.
struct PowerState {
  double* v;
  double* u;
  double* partials;
  GridBarrier bar;
};

struct ScaledGather {
  const double* v;
  double inv;
  __device__ __forceinline__ void add(double (&s)[1], double a, int k) const { s[0] += a * (ld(v + k) * inv); }
  __device__ __forceinline__ double product(int, double a, int k) const { return a * (ld(v + k) * inv); }
};

template <class T>
__global__ void __launch_bounds__(kThreads, 2) power_kernel(Prob<T> P, PowerState W, int iterations,
                                                            double* out) {
  __shared__ double sh[kWarps * 2];
  double* stream = warp_stream();
  const int G = gridDim.x, stride = G * kThreads;
  const int gt = blockIdx.x * kThreads + threadIdx.x;
  // ||v||^2 of the random start
  double a0[1] = {0.0};
  for (int j = gt; j < P.n; j += stride) {
    const double t = __ldcg(W.v + j);
    a0[0] += t * t;
  }
  block_reduce<1, 0u>(a0, sh);
  write_partials(W.partials, 0, a0, 1);
  if (!grid_barrier(W.bar)) return;
  for (int step = 0; step < iterations; ++step) {
    double len2[1];
    reduce_partials<1, 0u>(W.partials + (size_t)(step & 1) * G * kPartSlots, 0, len2, sh);
    const double length = sqrt(len2[0]);
    if (length == 0.0) {
      if (blockIdx.x == 0 && threadIdx.x == 0) *out = 1.0;
      return;
    }
    double dummy[1] = {0.0};
    run_phase<1, 1>(P.A.ptr, P.A.idx, P.A.val64, P.pa, ScaledGather{W.v, 1.0 / length},
                    StoreRow<1>{W.u, -1}, dummy, stream);
    if (!grid_barrier(W.bar)) return;
    double nx[1] = {0.0};
    run_phase<1, 1>(P.AT.ptr, P.AT.idx, P.AT.val64, P.pat, ScaledGather{W.u, 1.0},
                    StoreRow<1>{W.v, 0}, nx, stream);
    block_reduce<1, 0u>(nx, sh);
    write_partials(W.partials + (size_t)((step + 1) & 1) * G * kPartSlots, 0, nx, 1);
    if (!grid_barrier(W.bar)) return;
  }
  double fin[1];
  reduce_partials<1, 0u>(W.partials + (size_t)(iterations & 1) * G * kPartSlots, 0, fin, sh);
  const double norm = sqrt(sqrt(fin[0]));
  if (blockIdx.x == 0 && threadIdx.x == 0) *out = norm > 0.0 ? norm * 1.01 : 1.0;
}

}  // namespace sih26
