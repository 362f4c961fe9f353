// Device helpers shared by the PDHG kernels: bound tests, projection, warp/block reductions
// and a bounded grid barrier for cooperative launches.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sih26 {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;

// An absent bound is +-inf or any |v| >= 1e30; anything else (NaN included) is a finite bound
// (is_finite_bound, include/sankhya/types.hpp:32-39).
__device__ __forceinline__ bool finite_bound(double v) { return !(fabs(v) >= 1e30); }

// Host side: puts the calling thread's current device back when an entry point that switched
// to its own device returns, so a call never changes the device the caller works on.
struct DeviceGuard {
  int saved = -1;
  DeviceGuard() {
    if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
  }
  ~DeviceGuard() {
    int now = -1;
    if (saved >= 0 && cudaGetDevice(&now) == cudaSuccess && now != saved) cudaSetDevice(saved);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

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

// Grid-wide barrier for a cooperative launch (all blocks co-resident), on one word. Thread 0
// of each block adds to the word with an acq_rel atomic: block 0 adds 2^31 - (G - 1), every
// other block adds 1, so the word's top bit flips exactly when the last block arrives and
// its low 31 bits return to zero. The last arriver learns it from its own atomic; the others
// poll the word with acquire loads until the top bit differs from the value their atomic
// returned. bar.sync on either side extends the ordering to every thread of the block, so
// every write before the barrier is visible to every read after it. One atomic round trip
// for the last arriver, one poll after the flip for the others.
//
// Waiters give up after `limit_ns` (or as soon as another block has given up): they record an
// error and return false instead of waiting on, so a broken launch ends instead of hanging
// the GPU. A block that passed a barrier while another gave up stops at the next one, where
// its own wait sees the error word. A test can make the give-up path run: `skip_block` names
// a block that returns from the barrier without arriving (the host sets it only when the
// SANKHYA_PDHG_TEST_BARRIER_FAULT environment variable asks for it).
struct GridBarrier {
  unsigned* count;                  // the barrier word; zero before the first barrier
  int* error;
  unsigned long long limit_ns;
  int* time_up;                     // set by the last arriver: global time > deadline_ns
  unsigned long long deadline_ns;   // 0 = no deadline
  int skip_block;                   // fault injection (tests): this block never arrives; -1 none
};

__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed(unsigned* p, unsigned v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ bool grid_barrier(const GridBarrier& b) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0 && (int)blockIdx.x == b.skip_block) {
    ok = 0;  // the injected fault: this block stays away and the others give up
  } else if (threadIdx.x == 0) {
    const unsigned add = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1u) : 1u;
    const unsigned old = atom_add_acq_rel(b.count, add);
    int good = 1;
    if (((old ^ (old + add)) & 0x80000000u) != 0u) {
      // the last arriver
      if (b.deadline_ns != 0ull && global_ns() > b.deadline_ns)
        st_relaxed(reinterpret_cast<unsigned*>(b.time_up), 1u);
    } else {
      const unsigned long long t0 = global_ns();
      unsigned spins = 0;
      while (((ld_acquire(b.count) ^ old) & 0x80000000u) == 0u) {
        ++spins;
        if (spins > 4096) __nanosleep(32);
        if ((spins & 1023u) == 0) {
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
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

}  // namespace sih26
