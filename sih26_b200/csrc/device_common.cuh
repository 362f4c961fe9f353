// Device helpers shared by the PDHG kernels: bound tests, projection, warp/block reductions
// and a bounded grid barrier for cooperative launches.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sih26 {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;

// An absent bound is +-inf or any |v| >= 1e30 (include/sankhya/types.hpp:32-39).
__device__ __forceinline__ bool finite_bound(double v) { return fabs(v) < 1e30; }

// Componentwise projection onto [lo, hi], tolerant of infinite sides (src/pdhg/pdhg.cpp:63-67).
__device__ __forceinline__ double project(double v, double lo, double hi) {
  if (finite_bound(lo) && v < lo) return lo;
  if (finite_bound(hi) && v > hi) return hi;
  return v;
}

__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Reduction of NS slots over one warp. Bit i of MAXMASK selects max instead of sum for
// slot i. The xor tree is fixed, so the result is deterministic.
template <int NS, unsigned MAXMASK>
__device__ __forceinline__ void warp_reduce(double (&v)[NS]) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double o = __shfl_xor_sync(0xffffffffu, v[s], off);
      v[s] = ((MAXMASK >> s) & 1u) ? dmax(v[s], o) : v[s] + o;
    }
  }
}

// Block reduction of NS slots; every thread returns with the block total in v. Uses
// shared[kWarps * NS]. Fixed order: warp totals combined in warp order.
template <int NS, unsigned MAXMASK>
__device__ __forceinline__ void block_reduce(double (&v)[NS], double* shared) {
  warp_reduce<NS, MAXMASK>(v);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) shared[warp * NS + s] = v[s];
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double t = shared[s];
    for (int w = 1; w < kWarps; ++w) {
      const double o = shared[w * NS + s];
      t = ((MAXMASK >> s) & 1u) ? dmax(t, o) : t + o;
    }
    v[s] = t;
  }
  __syncthreads();
}

// Grid-wide barrier for a cooperative launch (all blocks co-resident). Thread 0 of each
// block arrives on a counter; the last arriver resets it and bumps the generation. Waiters
// spin on the generation with a deadline: after `limit_ns` they record an error and return
// false instead of waiting on, so a broken launch ends instead of hanging the GPU. The
// fences make every write before the barrier visible to every read after it (the same
// bar.sync / fence / atomic pattern as cooperative groups' grid sync).
struct GridBarrier {
  unsigned* count;
  unsigned* generation;
  int* error;
  unsigned long long limit_ns;
  int* time_up;                     // set by the last arriver: global time > deadline_ns
  unsigned long long deadline_ns;   // 0 = no deadline
};

__device__ __forceinline__ bool grid_barrier(const GridBarrier& b) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = b.generation;
    const unsigned g = *gen;
    __threadfence();
    const unsigned arrived = atomicAdd(b.count, 1u);
    int good = 1;
    if (arrived == gridDim.x - 1) {
      if (b.deadline_ns != 0ull && global_ns() > b.deadline_ns) atomicExch(b.time_up, 1);
      atomicExch(b.count, 0u);
      __threadfence();
      atomicAdd(b.generation, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      unsigned spins = 0;
      while (*gen == g) {
        if (++spins > 64) __nanosleep(64);
        if ((spins & 255u) == 0) {
          if (*((volatile int*)b.error) != 0) {  // another block already gave up
            good = 0;
            break;
          }
          if (global_ns() - t0 > b.limit_ns) {
            atomicExch(b.error, 1);
            good = 0;
            break;
          }
        }
      }
    }
    __threadfence();
    ok = good && (*((volatile int*)b.error) == 0);
  }
  __syncthreads();
  return ok != 0;
}

}  // namespace sih26
