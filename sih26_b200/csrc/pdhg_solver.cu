// The GPU restarted-PDHG solve behind the C ABI (include/sankhya_pdhg_gpu.h): host
// orchestration of the kernels in pdhg_kernels.cuh.
//
// Replaces sankhya::pdhg::solve_pdhg (src/pdhg/pdhg.cpp:267-726). Setup (validation, scaling,
// permutation, upload, norm estimate) runs once; the iteration loop then runs on the device
// in chunks of cooperative launches, the host reading one control block per chunk.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "pdhg_host.cuh"
#include "pdhg_kernels.cuh"
#include "prep_kernels.cuh"
#include "sankhya_pdhg_gpu.h"

namespace sih26 {

thread_local std::string g_last_error;

#define SIH26_CUDA(expr, code)                                                           \
  do {                                                                                   \
    const cudaError_t e_ = (expr);                                                       \
    if (e_ != cudaSuccess)                                                               \
      throw Failure{code, std::string(#expr) + ": " + cudaGetErrorString(e_)};           \
  } while (0)

using Clock = std::chrono::steady_clock;
static double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

// Owns every device allocation of one solve and counts the bytes it copies. Buffers are
// carved, 256-byte aligned, out of a few large cudaMalloc chunks (one call per 64 MiB or per
// larger buffer), so a solve's ~60 buffers cost a handful of allocations.
class Arena {
 public:
  long long h2d_bytes = 0;
  long long d2h_bytes = 0;
  ~Arena() {
    for (void* p : ptrs_) cudaFree(p);
  }
  template <class T>
  T* alloc(size_t count) {
    if (count == 0) count = 1;
    const size_t bytes = (count * sizeof(T) + 255) & ~size_t(255);
    if (bytes > left_) {
      constexpr size_t kChunk = size_t(64) << 20;
      const size_t size = std::max(bytes, kChunk);
      void* p = nullptr;
      SIH26_CUDA(cudaMalloc(&p, size), SANKHYA_GPU_OUT_OF_MEMORY);
      ptrs_.push_back(p);
      next_ = static_cast<unsigned char*>(p);
      left_ = size;
    }
    void* p = next_;
    next_ += bytes;
    left_ -= bytes;
    return static_cast<T*>(p);
  }
  // The stream every later use of the arena's buffers is ordered on: zeroing goes there too,
  // so a kernel on that stream never overtakes the memset of a buffer it reads (a
  // non-blocking stream does not wait for the legacy default stream).
  void set_stream(cudaStream_t s) { stream_ = s; }
  cudaStream_t stream() const { return stream_; }
  template <class T>
  T* zeros(size_t count) {
    T* p = alloc<T>(count);
    SIH26_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(count, 1) * sizeof(T), stream_),
               SANKHYA_GPU_COPY_FAILED);
    return p;
  }
  template <class T, class U>
  T* upload(const std::vector<U>& host) {
    T* p = alloc<T>(host.size());
    if (!host.empty()) {
      std::vector<T> conv(host.begin(), host.end());
      SIH26_CUDA(cudaMemcpyAsync(p, conv.data(), conv.size() * sizeof(T), cudaMemcpyHostToDevice,
                                 stream_), SANKHYA_GPU_COPY_FAILED);
      h2d_bytes += conv.size() * sizeof(T);
    }
    return p;
  }
  template <class T>
  T* upload_same(const std::vector<T>& host) {
    T* p = alloc<T>(host.size());
    if (!host.empty()) {
      SIH26_CUDA(cudaMemcpyAsync(p, host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice,
                                 stream_), SANKHYA_GPU_COPY_FAILED);
      h2d_bytes += host.size() * sizeof(T);
    }
    return p;
  }
  // host -> device copy of a plain buffer, counted
  void put(void* dst, const void* src, size_t bytes, cudaStream_t stream) {
    if (bytes == 0) return;
    SIH26_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream), SANKHYA_GPU_COPY_FAILED);
    h2d_bytes += bytes;
  }
  void get(void* dst, const void* src, size_t bytes, cudaStream_t stream) {
    if (bytes == 0) return;
    SIH26_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream), SANKHYA_GPU_COPY_FAILED);
    d2h_bytes += bytes;
  }

 private:
  std::vector<void*> ptrs_;
  unsigned char* next_ = nullptr;
  size_t left_ = 0;
  cudaStream_t stream_ = nullptr;
};

template <class T>
static std::vector<T> gather(const std::vector<T>& v, const std::vector<int>& perm) {
  std::vector<T> out(perm.size());
  for (size_t t = 0; t < perm.size(); ++t) out[t] = v[perm[t]];
  return out;
}
template <class T>
static std::vector<T> gather_ptr(const T* v, const std::vector<int>& perm) {
  std::vector<T> out(perm.size());
  for (size_t t = 0; t < perm.size(); ++t) out[t] = v[perm[t]];
  return out;
}

// Kernel launches of the current call on this thread (reported in the result).
thread_local long long g_launches = 0;

static Part upload_part(Arena& a, const HostPart& hp) {
  Part p;
  p.blk_seg_begin = a.upload_same(hp.blk_seg_begin);
  p.segs = a.upload_same(hp.segs);
  p.blk_long_begin = a.upload_same(hp.blk_long_begin);
  p.longs = a.upload_same(hp.longs);
  p.blk_item_begin = a.upload_same(hp.blk_item_begin);
  p.items = a.upload_same(hp.items);
  p.seg_sum = a.zeros<double>(hp.segs.size() * 2);
  p.sell_idx = nullptr;
  p.sell_val = nullptr;
  return p;
}

static dim3 fill_grid(size_t items) {
  return dim3(static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>((items + 7) / 8, 148 * 16))));
}

// A sliced partition (the iteration kernel's) with its slice arrays in value type T, filled on
// the device from the permuted CSR. `sidx` / `sval` may be given (scratch of at least
// hp.sell_entries entries, reused by the autotuner's candidates); else they are allocated.
template <class T>
static Part upload_sliced(Arena& a, const HostPart& hp, const int* ptr, const int* idx,
                          const double* val64, cudaStream_t stream, int* sidx = nullptr,
                          T* sval = nullptr) {
  Part p = upload_part(a, hp);
  const size_t entries = static_cast<size_t>(std::max<long long>(1, hp.sell_entries));
  if (!sidx) sidx = a.alloc<int>(entries);
  if (!sval) sval = a.alloc<T>(entries);
  const int count = static_cast<int>(hp.items.size());
  if (count > 0) {
    slice_fill_kernel<T><<<fill_grid(count), 256, 0, stream>>>(ptr, idx, val64, p.items, count,
                                                                sidx, sval);
    SIH26_CUDA(cudaGetLastError(), SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
    ++g_launches;
  }
  p.sell_idx = sidx;
  p.sell_val = sval;
  return p;
}


static void launch_coop(const void* fn, int grid, void** args, size_t smem, cudaStream_t stream) {
  SIH26_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, smem, stream),
             SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
  ++g_launches;
}

__global__ void read_clock_kernel(unsigned long long* out) { *out = global_ns(); }

// Everything one precision level of the solve needs on the device.
template <class T>
struct Level {
  Prob<T> P;
  State<T> S;
  bool halpern = false;  // which iteration kernel runs the loop
};

struct Common {
  // device copies shared by both precisions
  const int *a_ptr, *a_idx, *at_ptr, *at_idx;
  const double *a_val64, *at_val64;
  const double *dr, *dc, *c0, *cl0, *cu0, *rl0, *ru0;
  const double *c64, *cl64, *cu64, *rl64, *ru64;  // scaled, FP64
  Part pa, pat;
  double *best_x, *best_y, *cert_row, *cert_col, *partials;
  Ctrl* ctrl;
  GridBarrier bar;
};

template <class T>
static Level<T> make_level(Arena& a, const Common& cm, const PermutedLp& q,
                           const std::vector<double>& x0) {
  Level<T> L{};
  const int m = q.m, n = q.n;
  Prob<T>& P = L.P;
  P.m = m;
  P.n = n;
  P.A.ptr = cm.a_ptr;
  P.A.idx = cm.a_idx;
  P.A.val64 = cm.a_val64;
  P.AT.ptr = cm.at_ptr;
  P.AT.idx = cm.at_idx;
  P.AT.val64 = cm.at_val64;
  if constexpr (std::is_same<T, double>::value) {
    P.A.val = cm.a_val64;
    P.AT.val = cm.at_val64;
  } else {
    // FP32 copies of the scaled values, rounded on the device
    T* av = a.alloc<T>(q.nnz);
    T* atv = a.alloc<T>(q.nnz);
    const dim3 grid(static_cast<unsigned>(std::max<long long>(1, std::min<long long>((q.nnz + 255) / 256, 148 * 16))));
    prep::to_float<<<grid, 256, 0, a.stream()>>>(cm.a_val64, q.nnz, av);
    prep::to_float<<<grid, 256, 0, a.stream()>>>(cm.at_val64, q.nnz, atv);
    SIH26_CUDA(cudaGetLastError(), SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
    SIH26_CUDA(cudaDeviceSynchronize(), SANKHYA_GPU_SYNC_FAILED);
    P.A.val = av;
    P.AT.val = atv;
  }
  P.pa = cm.pa;
  P.pat = cm.pat;
  P.c64 = cm.c64;
  P.cl64 = cm.cl64;
  P.cu64 = cm.cu64;
  P.rl64 = cm.rl64;
  P.ru64 = cm.ru64;
  if constexpr (std::is_same<T, double>::value) {
    P.c = cm.c64;
    P.cl = cm.cl64;
    P.cu = cm.cu64;
    P.rl = cm.rl64;
    P.ru = cm.ru64;
  }
  P.dr = cm.dr;
  P.dc = cm.dc;
  P.c0 = cm.c0;
  P.cl0 = cm.cl0;
  P.cu0 = cm.cu0;
  P.rl0 = cm.rl0;
  P.ru0 = cm.ru0;
  State<T>& S = L.S;
  for (int k = 0; k < 2; ++k) {
    S.x[k] = a.zeros<T>(n);
    S.y[k] = a.zeros<T>(m);
    S.ax[k] = a.zeros<double>(m);
  }
  S.xsum = a.zeros<double>(n);
  S.ysum = a.zeros<double>(m);
  S.xr = a.zeros<double>(n);
  S.yr = a.zeros<double>(m);
  S.xc = a.zeros<double2>(n);
  S.yc = a.zeros<double2>(m);
  S.axr = a.zeros<double>(m);
  S.xt = a.zeros<T>(n);
  S.yt = a.zeros<T>(m);
  if constexpr (kDelta<T>) {
    S.cg = a.zeros<double>(n);
    S.dl = a.zeros<float>(n);
    S.du = a.zeros<float>(n);
  }
  S.best_x = cm.best_x;
  S.best_y = cm.best_y;
  S.cert_row = cm.cert_row;
  S.cert_col = cm.cert_col;
  S.partials = cm.partials;
  S.ctrl = cm.ctrl;
  S.bar = cm.bar;
  if (!x0.empty()) {
    // the FP64 level starts at x0; the FP32 level at the anchor x0 with zero deltas
    if constexpr (!kDelta<T>) a.put(S.x[0], x0.data(), n * sizeof(double), a.stream());
    a.put(S.xr, x0.data(), n * sizeof(double), a.stream());
    SIH26_CUDA(cudaDeviceSynchronize(), SANKHYA_GPU_SYNC_FAILED);
  }
  return L;
}

// Opts every kernel into its dynamic shared memory and returns how many blocks of each fit
// on an SM (the minimum over the kernels, which share one work partition).
template <class T>
static int blocks_per_sm() {
  // the iteration kernels run sliced partitions without a stream buffer: no dynamic shared
  // memory, and the whole on-chip memory they can have goes to L1 (the gathers' cache)
  int best = 1 << 20;
  for (const void* f : {reinterpret_cast<const void*>(iterate_kernel<T, false>),
                        reinterpret_cast<const void*>(iterate_kernel<T, true>)}) {
    SIH26_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    (int)cudaSharedmemCarveoutMaxL1), SANKHYA_GPU_INIT_FAILED);
    int b = 0;
    SIH26_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, kThreads, 0),
               SANKHYA_GPU_INIT_FAILED);
    best = std::min(best, b);
  }
  const void* k1[] = {reinterpret_cast<const void*>(init_ax_kernel<T>),
                      reinterpret_cast<const void*>(anchor_kernel<T>),
                      reinterpret_cast<const void*>(report_kernel<T>),
                      reinterpret_cast<const void*>(power_kernel<T>),
                      reinterpret_cast<const void*>(probe_kernel<T>)};
  for (const void* f : k1) {
    SIH26_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)stream_smem_bytes()), SANKHYA_GPU_INIT_FAILED);
    int b = 0;
    SIH26_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, f, kThreads, stream_smem_bytes()),
               SANKHYA_GPU_INIT_FAILED);
    best = std::min(best, b);
  }
  const void* ek = reinterpret_cast<const void*>(evaluate_kernel<T>);
  SIH26_CUDA(cudaFuncSetAttribute(ek, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)stream_smem_bytes()), SANKHYA_GPU_INIT_FAILED);
  int b = 0;
  SIH26_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, ek, kThreads, stream_smem_bytes()),
             SANKHYA_GPU_INIT_FAILED);
  return std::min(best, b);
}

// Per-device facts that do not change while the process runs: the properties and how many
// blocks of each level's kernels fit on an SM. The queries (and the shared-memory opt-ins)
// cost milliseconds -- most of the setup of a small LP -- so they run once per device.
struct DeviceFacts {
  cudaDeviceProp props{};
  int bpsm_fp64 = 0, bpsm_fp32 = 0;
};
static const DeviceFacts& device_facts(int device) {
  static std::mutex mu;
  static std::map<int, std::unique_ptr<DeviceFacts>> cache;
  std::lock_guard<std::mutex> lock(mu);
  std::unique_ptr<DeviceFacts>& slot = cache[device];
  if (!slot) {
    auto f = std::make_unique<DeviceFacts>();
    SIH26_CUDA(cudaGetDeviceProperties(&f->props, device), SANKHYA_GPU_INIT_FAILED);
    if (f->props.major >= 10) {
      f->bpsm_fp64 = blocks_per_sm<double>();
      f->bpsm_fp32 = blocks_per_sm<float>();
    }
    slot = std::move(f);
  }
  return *slot;
}

// Runs (iterate, evaluate) launch pairs until the device reports a final state. With
// Event-timed launches of the iteration kernel (profile_kernels).
struct LaunchTimer {
  bool on = false;
  std::vector<cudaEvent_t> start, stop;
  double seconds = 0.0;
  long long launches = 0;
  ~LaunchTimer() {
    for (auto e : start) cudaEventDestroy(e);
    for (auto e : stop) cudaEventDestroy(e);
  }
  void ensure(size_t k) {
    while (start.size() < k) {
      cudaEvent_t a, b;
      SIH26_CUDA(cudaEventCreate(&a), SANKHYA_GPU_INIT_FAILED);
      SIH26_CUDA(cudaEventCreate(&b), SANKHYA_GPU_INIT_FAILED);
      start.push_back(a);
      stop.push_back(b);
    }
  }
  void collect(int k) {
    for (int i = 0; i < k; ++i) {
      float ms = 0.f;
      SIH26_CUDA(cudaEventElapsedTime(&ms, start[i], stop[i]), SANKHYA_GPU_SYNC_FAILED);
      seconds += ms * 1e-3;
      ++launches;
    }
  }
};

// Runs (iterate, evaluate) launch pairs until the device reports a final state. With
// `stall_checks` > 0 (the FP32 phase of the mixed mode) it also returns, with *stalled set,
// once the best KKT error has not moved over that many host checks of at least 16 pairs each:
// the FP32 iterate has reached what its precision allows. kAutoStall is the default rule:
// no 1 % improvement over the last 30 % of the iterations, and over 8 checks at least --
// wide enough for the long plateaus restarted PDHG goes through on its own.
constexpr int kAutoStall = -2;

template <class T>
static Ctrl run_loop(Level<T>& L, int G, cudaStream_t stream, Ctrl* host_ctrl, int verbose,
                     int stall_checks, bool* stalled, LaunchTimer& timer) {
  long long max_attempts = 1ll << 40;
  int pairs = 4;
  Ctrl c{};
  double last_best = INFINITY;
  int flat = 0;
  double mark_best = INFINITY;     // auto rule: best error at the last 1 % improvement
  long long mark_iteration = 0;    // and the iteration it was seen at
  if (stalled) *stalled = false;
  for (;;) {
    if (timer.on) timer.ensure(pairs);
    for (int k = 0; k < pairs; ++k) {
      void* ia[] = {&L.P, &L.S, &max_attempts};
      if (timer.on) SIH26_CUDA(cudaEventRecord(timer.start[k], stream), SANKHYA_GPU_INIT_FAILED);
      launch_coop(L.halpern ? reinterpret_cast<const void*>(iterate_kernel<T, true>)
                            : reinterpret_cast<const void*>(iterate_kernel<T, false>),
                  G, ia, 0, stream);
      if (timer.on) SIH26_CUDA(cudaEventRecord(timer.stop[k], stream), SANKHYA_GPU_INIT_FAILED);
      void* ea[] = {&L.P, &L.S};
      launch_coop(reinterpret_cast<const void*>(evaluate_kernel<T>), G, ea, stream_smem_bytes(), stream);
    }
    SIH26_CUDA(cudaMemcpyAsync(host_ctrl, L.S.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, stream),
               SANKHYA_GPU_COPY_FAILED);
    SIH26_CUDA(cudaStreamSynchronize(stream), SANKHYA_GPU_SYNC_FAILED);
    if (timer.on) timer.collect(pairs);
    c = *host_ctrl;
    if (verbose) {
      std::printf("%10lld %12.5e %10.3e %10.3e %10.3e %9.2e %9.2e %s\n", c.iteration,
                  c.best.primal_objective, c.best.primal, c.best.dual, c.best.gap, c.eta,
                  c.omega, sizeof(T) == 4 ? "fp32" : "fp64");
      std::fflush(stdout);
    }
    if (c.state != kRunning && c.state != kNeedEval) break;
    if (stall_checks > 0 && pairs >= 16) {
      flat = (c.best_worst >= last_best) ? flat + 1 : 0;
      if (flat >= stall_checks) {
        *stalled = true;
        break;
      }
    } else if (stall_checks == kAutoStall) {
      // no 1 % improvement over the last 30 % of the iterations (and 8 checks at least)
      if (c.best_worst < 0.99 * mark_best) {
        mark_best = c.best_worst;
        mark_iteration = c.iteration;
        flat = 0;
      } else if (pairs >= 16) {
        ++flat;
      }
      if (flat >= 8 && c.iteration - mark_iteration > (long long)(0.3 * (double)c.iteration)) {
        *stalled = true;
        break;
      }
    }
    last_best = c.best_worst;
    if (pairs < 64) pairs *= 2;
  }
  return c;
}

// A certificate the device found, checked on the host against the original problem.
struct Certificate {
  int kind = 0;               // 0 none, kInfeasible or kUnbounded
  std::vector<double> value;  // original order: Farkas multipliers [m] or a primal ray [n]
  int rejected = 0;           // candidates the exact check turned down
};

// run_loop, plus the host half of infeasibility detection: when the device stops on a
// certificate candidate, the candidate is copied back, un-permuted and checked with the
// reference's exact rules (farkas_holds / ray_holds). A proof ends the solve; anything else
// resumes the loop from the same state with the test paused for kCertCooldown evaluations.
template <class T>
static Ctrl run_loop_checked(Level<T>& L, int G, cudaStream_t stream, Ctrl* host_ctrl,
                             int verbose, int stall_checks, bool* stalled, LaunchTimer& timer,
                             const sankhya_pdhg_problem& prob, const PermutedLp& q, Arena& a,
                             const double* cert_row, const double* cert_col, Certificate& cert) {
  for (;;) {
    Ctrl c = run_loop(L, G, stream, host_ctrl, verbose, stall_checks, stalled, timer);
    if (c.state != kInfeasible && c.state != kUnbounded) return c;
    const bool rows = c.state == kInfeasible;
    const int len = rows ? q.m : q.n;
    std::vector<double> h(len), v(len);
    a.get(h.data(), rows ? cert_row : cert_col, len * sizeof(double), stream);
    SIH26_CUDA(cudaStreamSynchronize(stream), SANKHYA_GPU_SYNC_FAILED);
    const std::vector<int>& perm = rows ? q.row_perm : q.col_perm;
    for (int t = 0; t < len; ++t) v[perm[t]] = h[t];
    bool ok = rows ? farkas_holds(prob, v) : ray_holds(prob, v);
    if (!ok && !rows && repair_ray(prob, v)) ok = ray_holds(prob, v);
    if (ok) {
      cert.kind = c.state;
      cert.value = std::move(v);
      return c;
    }
    ++cert.rejected;
    c.state = kRunning;
    c.farkas_cooldown = kCertCooldown;
    a.put(L.S.ctrl, &c, sizeof(Ctrl), stream);
    if (kDelta<T> && !rows && stalled) {
      // the FP32 level sees a ray it cannot resolve to the checker's 1e-7: the FP64 level
      // takes over from here (the mixed mode's hand-over) and certifies it
      *stalled = true;
      return c;
    }
  }
}

// Relative KKT error below which the FP32 phase of the mixed mode hands over by default.
// FP32 deltas about an FP64 anchor keep their accuracy as the restarts close in (a plain FP32
// iterate stalls near 256 units of FP32 rounding, ~1.5e-5), so this is only a backstop for
// requests at the edge of FP64 itself; the stall rule catches a level that stops improving.
constexpr double kFp32Reach = 1e-10;

static int G_max_coresident(const cudaDeviceProp& props, int bpsm) {
  return props.multiProcessorCount * bpsm;
}

// ---- preparation on the device (prep_kernels.cuh) --------------------------------------

static int bits_for(long long count) {  // bits that hold 0 .. count-1
  int b = 1;
  while ((1ll << b) < count) ++b;
  return b;
}

static dim3 prep_grid(long long work) {
  return dim3(static_cast<unsigned>(std::max<long long>(1, std::min<long long>((work + 255) / 256, 148 * 16))));
}

template <class K, class V>
static void radix_sort_pairs(Arena& a, const K* kin, K* kout, const V* vin, V* vout, long long count,
                             int end_bit, cudaStream_t stream) {
  size_t bytes = 0;
  SIH26_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, count, 0, end_bit,
                                             stream), SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
  void* tmp = a.alloc<unsigned char>(bytes);
  SIH26_CUDA(cub::DeviceRadixSort::SortPairs(tmp, bytes, kin, kout, vin, vout, count, 0, end_bit,
                                             stream), SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
  g_launches += 1;
}

// ptr[0] = 0, ptr[i+1] = ptr[i] + len[i]
static void lengths_to_ptr(Arena& a, const int* len, int count, int* ptr, cudaStream_t stream) {
  SIH26_CUDA(cudaMemsetAsync(ptr, 0, sizeof(int), stream), SANKHYA_GPU_COPY_FAILED);
  if (count == 0) return;
  size_t bytes = 0;
  SIH26_CUDA(cub::DeviceScan::InclusiveSum(nullptr, bytes, len, ptr + 1, count, stream),
             SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
  void* tmp = a.alloc<unsigned char>(bytes);
  SIH26_CUDA(cub::DeviceScan::InclusiveSum(tmp, bytes, len, ptr + 1, count, stream),
             SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
  g_launches += 1;
}

// build_scaling + permute on the device: fills the device arrays of `cm` (matrix, scaling and
// vectors, permuted) and, on the host, q's sizes, permutations and row pointers (the work
// partition and the output un-permutation are built from them) and the starting point x0.
static void prepare_on_device(Arena& a, const sankhya_pdhg_problem& prob,
                              const std::vector<double>& cmin, int ruiz_rounds,
                              cudaStream_t stream, Common& cm, PermutedLp& q,
                              std::vector<double>& x0) {
  using namespace prep;
  const int m = prob.num_rows, n = prob.num_cols;
  const long long nnz = prob.num_nonzeros;
  q.m = m;
  q.n = n;
  q.nnz = nnz;
  const auto put_i = [&](const int* h, size_t count) {
    int* d = a.alloc<int>(count);
    a.put(d, h, count * sizeof(int), stream);
    return d;
  };
  const auto put_d = [&](const double* h, size_t count) {
    double* d = a.alloc<double>(count);
    a.put(d, h, count * sizeof(double), stream);
    return d;
  };
  const dim3 B(256);
  // the problem as given (CSC) and the entries' columns
  int* cs = put_i(prob.col_starts, n + 1);
  int* ri = put_i(prob.row_indices, nnz);
  double* v = put_d(prob.values, nnz);
  double* cmin_d = put_d(cmin.data(), n);
  double* cl = put_d(prob.col_lower, n);
  double* cu = put_d(prob.col_upper, n);
  double* rl = put_d(prob.row_lower, m);
  double* ru = put_d(prob.row_upper, m);
  int* col = a.alloc<int>(nnz);
  column_of_entry<<<prep_grid(n), B, 0, stream>>>(cs, n, col);
  // row-major copy: a stable sort of the entries by row keeps each row in column order
  int* rcount = a.zeros<int>(m);
  count_by<<<prep_grid(nnz), B, 0, stream>>>(ri, nnz, rcount);
  int* rptr = a.alloc<int>(m + 1);
  lengths_to_ptr(a, rcount, m, rptr, stream);
  int* entry = a.alloc<int>(nnz);
  int* entry_rm = a.alloc<int>(nnz);
  unsigned* rkey_in = a.alloc<unsigned>(nnz);
  unsigned* rkey_out = a.alloc<unsigned>(nnz);
  SIH26_CUDA(cudaMemcpyAsync(rkey_in, ri, nnz * sizeof(int), cudaMemcpyDeviceToDevice, stream),
             SANKHYA_GPU_COPY_FAILED);
  identity<<<prep_grid(nnz), B, 0, stream>>>(entry, nnz);
  radix_sort_pairs(a, rkey_in, rkey_out, entry, entry_rm, nnz, bits_for(m), stream);
  double* vr = a.alloc<double>(nnz);
  int* cr = a.alloc<int>(nnz);
  int* rr = a.alloc<int>(nnz);
  gather<double><<<prep_grid(nnz), B, 0, stream>>>(entry_rm, v, nnz, vr);
  gather<int><<<prep_grid(nnz), B, 0, stream>>>(entry_rm, col, nnz, cr);
  row_of_entry<<<prep_grid(m), B, 0, stream>>>(rptr, m, rr);
  // scaling rounds: 10 Ruiz (max) and one Pock-Chambolle (sum), scaling.cpp:44-100
  double* ra = a.alloc<double>(m);
  double* ca = a.alloc<double>(n);
  double* rp = a.alloc<double>(m);
  double* cp = a.alloc<double>(n);
  double* dr = a.alloc<double>(m);
  double* dc = a.alloc<double>(n);
  fill<<<prep_grid(m), B, 0, stream>>>(dr, m, 1.0);
  fill<<<prep_grid(n), B, 0, stream>>>(dc, n, 1.0);
  for (int round = 0; round <= ruiz_rounds; ++round) {
    const int sum = round == ruiz_rounds ? 1 : 0;
    segment_norms<<<prep_grid(n), B, 0, stream>>>(cs, v, n, sum, ca);
    segment_norms<<<prep_grid(m), B, 0, stream>>>(rptr, vr, m, sum, ra);
    pass_factors<<<prep_grid(m), B, 0, stream>>>(ra, m, rp, dr);
    pass_factors<<<prep_grid(n), B, 0, stream>>>(ca, n, cp, dc);
    apply_pass<<<prep_grid(nnz), B, 0, stream>>>(ri, col, rp, cp, nnz, v);
    apply_pass<<<prep_grid(nnz), B, 0, stream>>>(rr, cr, rp, cp, nnz, vr);
    g_launches += 6;
  }
  // scaled vectors, original order
  double* c_s = a.alloc<double>(n);
  double* cl_s = a.alloc<double>(n);
  double* cu_s = a.alloc<double>(n);
  double* rl_s = a.alloc<double>(m);
  double* ru_s = a.alloc<double>(m);
  scaled_columns<<<prep_grid(n), B, 0, stream>>>(cmin_d, cl, cu, dc, n, c_s, cl_s, cu_s);
  scaled_rows<<<prep_grid(m), B, 0, stream>>>(rl, ru, dr, m, rl_s, ru_s);
  // permutations: longest first, ties by index
  int* row_perm = a.alloc<int>(m);
  int* col_perm = a.alloc<int>(n);
  {
    unsigned* k_in = a.alloc<unsigned>(std::max(m, n));
    unsigned* k_out = a.alloc<unsigned>(std::max(m, n));
    int* idx = a.alloc<int>(std::max(m, n));
    count_keys<<<prep_grid(m), B, 0, stream>>>(rptr, m, k_in, idx);
    radix_sort_pairs(a, k_in, k_out, idx, row_perm, m, 32, stream);
    count_keys<<<prep_grid(n), B, 0, stream>>>(cs, n, k_in, idx);
    radix_sort_pairs(a, k_in, k_out, idx, col_perm, n, 32, stream);
  }
  int* row_pos = a.alloc<int>(m);
  int* col_pos = a.alloc<int>(n);
  positions<<<prep_grid(m), B, 0, stream>>>(row_perm, m, row_pos);
  positions<<<prep_grid(n), B, 0, stream>>>(col_perm, n, col_pos);
  // A in permuted row order, each row's entries in permuted column order; A' likewise
  int* a_ptr = a.alloc<int>(m + 1);
  int* at_ptr = a.alloc<int>(n + 1);
  int* lens = a.alloc<int>(std::max(m, n));
  permuted_lengths<<<prep_grid(m), B, 0, stream>>>(rptr, row_perm, m, lens);
  lengths_to_ptr(a, lens, m, a_ptr, stream);
  permuted_lengths<<<prep_grid(n), B, 0, stream>>>(cs, col_perm, n, lens);
  lengths_to_ptr(a, lens, n, at_ptr, stream);
  unsigned long long* key_in = a.alloc<unsigned long long>(nnz);
  unsigned long long* key_out = a.alloc<unsigned long long>(nnz);
  int* a_idx = a.alloc<int>(nnz);
  int* at_idx = a.alloc<int>(nnz);
  double* a_val = a.alloc<double>(nnz);
  double* at_val = a.alloc<double>(nnz);
  {
    const int shift = bits_for(n), end = shift + bits_for(m);
    pair_keys<<<prep_grid(nnz), B, 0, stream>>>(ri, col, row_pos, col_pos, nnz, shift, key_in);
    radix_sort_pairs(a, key_in, key_out, v, a_val, nnz, end, stream);
    low_bits<<<prep_grid(nnz), B, 0, stream>>>(key_out, nnz, shift, a_idx);
  }
  {
    const int shift = bits_for(m), end = shift + bits_for(n);
    pair_keys<<<prep_grid(nnz), B, 0, stream>>>(col, ri, col_pos, row_pos, nnz, shift, key_in);
    radix_sort_pairs(a, key_in, key_out, v, at_val, nnz, end, stream);
    low_bits<<<prep_grid(nnz), B, 0, stream>>>(key_out, nnz, shift, at_idx);
  }
  cm.a_ptr = a_ptr;
  cm.a_idx = a_idx;
  cm.at_ptr = at_ptr;
  cm.at_idx = at_idx;
  cm.a_val64 = a_val;
  cm.at_val64 = at_val;
  const auto perm_vec = [&](const int* perm, const double* src, int len) {
    double* d = a.alloc<double>(len);
    gather<double><<<prep_grid(len), B, 0, stream>>>(perm, src, len, d);
    return d;
  };
  cm.dr = perm_vec(row_perm, dr, m);
  cm.dc = perm_vec(col_perm, dc, n);
  cm.c0 = perm_vec(col_perm, cmin_d, n);
  cm.cl0 = perm_vec(col_perm, cl, n);
  cm.cu0 = perm_vec(col_perm, cu, n);
  cm.rl0 = perm_vec(row_perm, rl, m);
  cm.ru0 = perm_vec(row_perm, ru, m);
  cm.c64 = perm_vec(col_perm, c_s, n);
  cm.cl64 = perm_vec(col_perm, cl_s, n);
  cm.cu64 = perm_vec(col_perm, cu_s, n);
  cm.rl64 = perm_vec(row_perm, rl_s, m);
  cm.ru64 = perm_vec(row_perm, ru_s, m);
  double* x0_d = a.alloc<double>(n);
  start_point<<<prep_grid(n), B, 0, stream>>>(cm.cl64, cm.cu64, n, x0_d);
  SIH26_CUDA(cudaGetLastError(), SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
  // host copies the partition and the output un-permutation need
  q.row_perm.resize(m);
  q.col_perm.resize(n);
  q.a_ptr.resize(m + 1);
  q.at_ptr.resize(n + 1);
  x0.resize(n);
  a.get(q.row_perm.data(), row_perm, m * sizeof(int), stream);
  a.get(q.col_perm.data(), col_perm, n * sizeof(int), stream);
  a.get(q.a_ptr.data(), a_ptr, (m + 1) * sizeof(int), stream);
  a.get(q.at_ptr.data(), at_ptr, (n + 1) * sizeof(int), stream);
  a.get(x0.data(), x0_d, n * sizeof(double), stream);
  SIH26_CUDA(cudaStreamSynchronize(stream), SANKHYA_GPU_SYNC_FAILED);
}

// Mean microseconds of one probe SpMV over `part` (after one warm-up launch).
template <class T>
static double time_probe(const int* ptr, const int* idx, const T* val, const Part& part,
                         const T* v, double* out, int G, cudaStream_t stream, cudaEvent_t e0,
                         cudaEvent_t e1) {
  constexpr int kReps = 5;
  probe_kernel<T><<<G, kThreads, stream_smem_bytes(), stream>>>(ptr, idx, val, part, v, out);
  SIH26_CUDA(cudaEventRecord(e0, stream), SANKHYA_GPU_INIT_FAILED);
  for (int r = 0; r < kReps; ++r)
    probe_kernel<T><<<G, kThreads, stream_smem_bytes(), stream>>>(ptr, idx, val, part, v, out);
  SIH26_CUDA(cudaEventRecord(e1, stream), SANKHYA_GPU_INIT_FAILED);
  SIH26_CUDA(cudaGetLastError(), SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
  g_launches += kReps + 1;
  SIH26_CUDA(cudaEventSynchronize(e1), SANKHYA_GPU_SYNC_FAILED);
  float ms = 0.f;
  SIH26_CUDA(cudaEventElapsedTime(&ms, e0, e1), SANKHYA_GPU_SYNC_FAILED);
  return ms * 1e3 / kReps;
}

// The autotuner: for each orientation, the schedule (stream-row limit, nonzeros per lane)
// whose plain SpMV over this LP's matrix is fastest among a few candidates, at the level the
// iteration runs in. Results are keyed on row-length statistics and cached on disk, so LPs of
// the same shape family are tuned once.
template <class T>
static int autotune_schedules(Arena& a, const PermutedLp& q, const Level<T>& L, int G, int sms,
                              cudaStream_t stream, Schedule* sa, Schedule* sat) {
  const std::string key = autotune_key(q, G, sms, static_cast<int>(sizeof(T)));
  const std::string path = autotune_cache_path();
  if (autotune_lookup(path, key, sa, sat)) return 2;
  static const Schedule kCandidates[] = {{32, 16}, {16, 16}, {32, 8}, {32, 32}, {8, 16}, {16, 8}};
  double* out = a.zeros<double>(static_cast<size_t>(std::max(q.m, q.n)));
  cudaEvent_t e0, e1;
  SIH26_CUDA(cudaEventCreate(&e0), SANKHYA_GPU_INIT_FAILED);
  SIH26_CUDA(cudaEventCreate(&e1), SANKHYA_GPU_INIT_FAILED);
  struct EvFree {
    cudaEvent_t a, b;
    ~EvFree() { cudaEventDestroy(a); cudaEventDestroy(b); }
  } ef{e0, e1};
  double best_a = INFINITY, best_at = INFINITY;
  // the candidates' sliced partitions, and one scratch for their slice arrays per orientation
  std::vector<HostPart> ha, hat;
  long long ea = 1, eat = 1;
  for (const Schedule& c : kCandidates) {
    ha.push_back(partition(q.a_ptr, G, kWarps, 0, c, true));
    hat.push_back(partition(q.at_ptr, G, kWarps, 0, c, true));
    ea = std::max(ea, ha.back().sell_entries);
    eat = std::max(eat, hat.back().sell_entries);
  }
  int* sidx_a = a.alloc<int>(ea);
  T* sval_a = a.alloc<T>(ea);
  int* sidx_at = a.alloc<int>(eat);
  T* sval_at = a.alloc<T>(eat);
  for (size_t k = 0; k < ha.size(); ++k) {
    const Part pa = upload_sliced<T>(a, ha[k], L.P.A.ptr, L.P.A.idx, L.P.A.val64, stream,
                                     sidx_a, sval_a);
    const double ta = time_probe<T>(L.P.A.ptr, L.P.A.idx, L.P.A.val, pa, L.S.xt, out, G, stream, e0, e1);
    if (ta < best_a) {
      best_a = ta;
      *sa = kCandidates[k];
    }
    const Part pat = upload_sliced<T>(a, hat[k], L.P.AT.ptr, L.P.AT.idx, L.P.AT.val64, stream,
                                      sidx_at, sval_at);
    const double tat = time_probe<T>(L.P.AT.ptr, L.P.AT.idx, L.P.AT.val, pat, L.S.yt, out, G, stream, e0, e1);
    if (tat < best_at) {
      best_at = tat;
      *sat = kCandidates[k];
    }
  }
  autotune_store(path, key, *sa, *sat, best_a, best_at);
  return 1;
}

static void fill_message(sankhya_pdhg_result* r, const char* text) {
  std::snprintf(r->message, sizeof r->message, "%s", text);
}

static int solve_impl(const sankhya_pdhg_problem& prob, const sankhya_pdhg_params& prm,
                      sankhya_pdhg_result* res) {
  const Clock::time_point t_start = Clock::now();
  g_launches = 0;
  check_structure(prob);
  if (!(prm.tolerance > 0.0)) throw Failure{SANKHYA_GPU_INVALID_ARGUMENT, "tolerance must be > 0"};
  if (prm.precision != SANKHYA_PDHG_FP64 && prm.precision != SANKHYA_PDHG_MIXED)
    throw Failure{SANKHYA_GPU_INVALID_ARGUMENT, "unknown precision"};
  if (prm.algorithm != SANKHYA_PDHG_ALGORITHM_REFERENCE &&
      prm.algorithm != SANKHYA_PDHG_ALGORITHM_HALPERN)
    throw Failure{SANKHYA_GPU_INVALID_ARGUMENT, "unknown algorithm"};
  const int m = prob.num_rows, n = prob.num_cols;
  res->status = SANKHYA_PDHG_NOT_SOLVED;
  res->converged = 0;
  res->iterations = res->attempts = res->restarts = res->evaluations = res->fp32_iterations = 0;
  res->message[0] = '\0';
  const std::string why = validate_model(prob);
  if (!why.empty()) {
    res->status = SANKHYA_PDHG_MODEL_ERROR;
    fill_message(res, why.c_str());
    return SANKHYA_GPU_SUCCESS;
  }

  int devices = 0;
  if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0)
    throw Failure{SANKHYA_GPU_NO_COMPATIBLE_DEVICE, "no CUDA device is visible"};
  if (prm.device < 0 || prm.device >= devices)
    throw Failure{SANKHYA_GPU_INVALID_ARGUMENT, "device ordinal out of range"};
  SIH26_CUDA(cudaSetDevice(prm.device), SANKHYA_GPU_INIT_FAILED);
  const DeviceFacts& facts = device_facts(prm.device);
  const cudaDeviceProp& props = facts.props;
  if (props.major < 10)
    throw Failure{SANKHYA_GPU_NO_COMPATIBLE_DEVICE, "this library is built for sm_100a (B200)"};
  if (!props.cooperativeLaunch)
    throw Failure{SANKHYA_GPU_NO_COMPATIBLE_DEVICE, "device lacks cooperative launch"};

  // ---- the unscaled problem in minimise space (pdhg.cpp:284-301) ----
  const double sense = prob.maximize ? -1.0 : 1.0;
  std::vector<double> cmin(n);
  for (int j = 0; j < n; ++j) cmin[j] = sense * prob.cost[j];
  double cs2 = 0.0;
  for (int j = 0; j < n; ++j) cs2 += cmin[j] * cmin[j];
  const double cost_norm = std::sqrt(cs2);
  double bs2 = 0.0;
  for (int i = 0; i < m; ++i) {
    const double b = host_finite_bound(prob.row_lower[i])
                         ? prob.row_lower[i]
                         : (host_finite_bound(prob.row_upper[i]) ? prob.row_upper[i] : 0.0);
    bs2 += b * b;
  }
  const double bound_norm = std::sqrt(bs2);

  // setup phases, printed with the iteration table (verbose)
  std::vector<std::pair<const char*, double>> marks;
  const auto mark = [&](const char* what) { marks.emplace_back(what, seconds_since(t_start)); };
  mark("validation");

  // ---- preconditioning and layout ----
  int bpsm = std::min(facts.bpsm_fp64, prm.precision == SANKHYA_PDHG_MIXED ? facts.bpsm_fp32 : 1 << 20);
  if (bpsm < 1) throw Failure{SANKHYA_GPU_INIT_FAILED, "kernel does not fit on an SM"};
  int G = props.multiProcessorCount * std::min(bpsm, 2);
  const long long work = static_cast<long long>(prob.num_nonzeros) + m + n;
  G = static_cast<int>(std::max<long long>(1, std::min<long long>(G, (work + 4095) / 4096)));
  if (prm.grid_blocks > 0) G = std::min(G_max_coresident(props, bpsm), prm.grid_blocks);

  cudaStream_t stream;
  SIH26_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), SANKHYA_GPU_INIT_FAILED);
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{stream};
  Arena a;  // destroyed before the stream (declared after it)
  a.set_stream(stream);

  Common cm{};
  PermutedLp q;           // host: sizes, permutations, row pointers of A and A'
  std::vector<double> x0;  // the starting point, permuted
  constexpr long long kDevicePrepMinNnz = 100000;
  const bool host_prep = prm.prep == 1 || (prm.prep == 0 && prob.num_nonzeros < kDevicePrepMinNnz);
  if (host_prep) {
    // build_scaling and permute on the host (pdhg_host.cpp), uploaded
    const Scaling sc = build_scaling(prob, cmin, 10);
    q = permute(prob, sc.values);
    cm.a_ptr = a.upload_same(q.a_ptr);
    cm.a_idx = a.upload_same(q.a_idx);
    cm.at_ptr = a.upload_same(q.at_ptr);
    cm.at_idx = a.upload_same(q.at_idx);
    cm.a_val64 = a.upload_same(q.a_val);
    cm.at_val64 = a.upload_same(q.at_val);
    cm.dr = a.upload_same(gather(sc.dr, q.row_perm));
    cm.dc = a.upload_same(gather(sc.dc, q.col_perm));
    cm.c0 = a.upload_same(gather(cmin, q.col_perm));
    cm.cl0 = a.upload_same(gather_ptr(prob.col_lower, q.col_perm));
    cm.cu0 = a.upload_same(gather_ptr(prob.col_upper, q.col_perm));
    cm.rl0 = a.upload_same(gather_ptr(prob.row_lower, q.row_perm));
    cm.ru0 = a.upload_same(gather_ptr(prob.row_upper, q.row_perm));
    cm.c64 = a.upload_same(gather(sc.cost, q.col_perm));
    cm.cl64 = a.upload_same(gather(sc.cl, q.col_perm));
    cm.cu64 = a.upload_same(gather(sc.cu, q.col_perm));
    cm.rl64 = a.upload_same(gather(sc.rl, q.row_perm));
    cm.ru64 = a.upload_same(gather(sc.ru, q.row_perm));
    // starting point: the projection of zero (pdhg.cpp:329-334), in permuted order
    x0.resize(n);
    for (int t = 0; t < n; ++t) {
      const int j = q.col_perm[t];
      double v = 0.0;
      if (host_finite_bound(sc.cl[j]) && v < sc.cl[j]) v = sc.cl[j];
      else if (host_finite_bound(sc.cu[j]) && v > sc.cu[j]) v = sc.cu[j];
      x0[t] = v;
    }
  } else {
    prepare_on_device(a, prob, cmin, 10, stream, cm, q, x0);
  }
  mark("scaling and layout");
  cm.pa = upload_part(a, partition(q.a_ptr, G, kWarps, prm.group_size_rows));
  cm.pat = upload_part(a, partition(q.at_ptr, G, kWarps, prm.group_size_cols));
  cm.best_x = a.zeros<double>(n);
  cm.best_y = a.zeros<double>(m);
  cm.cert_row = a.zeros<double>(m);
  cm.cert_col = a.zeros<double>(n);
  cm.partials = a.zeros<double>(2ull * G * kPartSlots);
  cm.ctrl = a.zeros<Ctrl>(1);
  unsigned* bar_words = a.zeros<unsigned>(2);
  int* flags = a.zeros<int>(2);
  cm.bar = GridBarrier{bar_words, flags, 4000000000ull, flags + 1, 0ull, -1};
  a.put(cm.best_x, x0.data(), n * sizeof(double), stream);
  SIH26_CUDA(cudaDeviceSynchronize(), SANKHYA_GPU_SYNC_FAILED);

  mark("work partition");
  Level<double> L64 = make_level<double>(a, cm, q, prm.precision == SANKHYA_PDHG_FP64 ? x0 : std::vector<double>());
  Level<float> L32{};
  const bool mixed = prm.precision == SANKHYA_PDHG_MIXED;
  if (mixed) L32 = make_level<float>(a, cm, q, x0);

  // SpMV schedules: the fixed rule, or the autotuner's pick at the level the loop starts in
  Schedule sched_a, sched_at;
  int autotuned = 0;
  mark("iterate buffers");
  if (prm.autotune && prm.group_size_rows <= 0 && prm.group_size_cols <= 0 && q.nnz > 0) {
    autotuned = mixed ? autotune_schedules(a, q, L32, G, props.multiProcessorCount, stream,
                                           &sched_a, &sched_at)
                      : autotune_schedules(a, q, L64, G, props.multiProcessorCount, stream,
                                           &sched_a, &sched_at);
    cm.pa = upload_part(a, partition(q.a_ptr, G, kWarps, 0, sched_a));
    cm.pat = upload_part(a, partition(q.at_ptr, G, kWarps, 0, sched_at));
    L64.P.pa = L32.P.pa = cm.pa;
    L64.P.pat = L32.P.pat = cm.pat;
  }

  // the iteration kernel's sliced partitions with the same schedule, and their slice arrays
  // (column indices shared by both levels, values in each level's type)
  {
    const HostPart hai = partition(q.a_ptr, G, kWarps, prm.group_size_rows, sched_a, true);
    const HostPart hati = partition(q.at_ptr, G, kWarps, prm.group_size_cols, sched_at, true);
    L64.P.pai = upload_sliced<double>(a, hai, cm.a_ptr, cm.a_idx, cm.a_val64, stream);
    L64.P.pati = upload_sliced<double>(a, hati, cm.at_ptr, cm.at_idx, cm.at_val64, stream);
    if (mixed) {
      L32.P.pai = upload_sliced<float>(a, hai, cm.a_ptr, cm.a_idx, cm.a_val64, stream,
                                       const_cast<int*>(L64.P.pai.sell_idx));
      L32.P.pati = upload_sliced<float>(a, hati, cm.at_ptr, cm.at_idx, cm.at_val64, stream,
                                        const_cast<int*>(L64.P.pati.sell_idx));
    }
    // both levels evaluate over the FP64 slices
    L64.P.pae = L32.P.pae = L64.P.pai;
    L64.P.pate = L32.P.pate = L64.P.pati;
  }
  mark("schedules");
  // ||A||_2 by power iteration (scaling.cpp:161-194), seed random_seed + 1
  double spectral_norm = 1.0;
  if (m > 0 && n > 0 && q.nnz > 0) {
    std::vector<double> v0(n);
    uniform_draws(static_cast<uint32_t>(prm.random_seed) + 1u, -1.0, 1.0, n, v0.data());
    PowerState W{a.upload_same(gather(v0, q.col_perm)), a.zeros<double>(m), cm.partials, cm.bar};
    double* d_norm = a.zeros<double>(1);
    int iters = 30;
    void* pa[] = {&L64.P, &W, &iters, &d_norm};
    launch_coop(reinterpret_cast<const void*>(power_kernel<double>), G, pa, stream_smem_bytes(), stream);
    SIH26_CUDA(cudaMemcpyAsync(&spectral_norm, d_norm, sizeof(double), cudaMemcpyDeviceToHost, stream),
               SANKHYA_GPU_COPY_FAILED);
  }
  // A x0 for the starting point, with the same phase code as the iteration's A x'
  const bool halpern = prm.algorithm == SANKHYA_PDHG_ALGORITHM_HALPERN;
  if (mixed) {
    anchor_kernel<float><<<G, kThreads, stream_smem_bytes(), stream>>>(L32.P, L32.S);
  } else {
    init_ax_kernel<double><<<G, kThreads, stream_smem_bytes(), stream>>>(L64.P, L64.S);
    // the Halpern operator's A x_0 for the starting point (x_0 = x0)
    if (halpern)
      SIH26_CUDA(cudaMemcpyAsync(L64.S.axr, L64.S.ax[0], m * sizeof(double),
                                 cudaMemcpyDeviceToDevice, stream), SANKHYA_GPU_COPY_FAILED);
  }
  SIH26_CUDA(cudaGetLastError(), SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
  ++g_launches;
  int err_flag = 0;
  SIH26_CUDA(cudaStreamSynchronize(stream), SANKHYA_GPU_SYNC_FAILED);
  SIH26_CUDA(cudaMemcpy(&err_flag, flags, sizeof(int), cudaMemcpyDeviceToHost), SANKHYA_GPU_COPY_FAILED);
  if (err_flag) throw Failure{SANKHYA_GPU_DEVICE_TIMEOUT, "grid barrier timed out in the norm estimate"};

  const long long iteration_limit = prm.iteration_limit < 0 ? 1000000ll : prm.iteration_limit;
  Ctrl c0{};
  c0.eta = spectral_norm > 0.0 ? 1.0 / spectral_norm : 1.0;
  c0.omega = 1.0;
  c0.restart_kkt = INFINITY;
  c0.best_worst = INFINITY;
  c0.best.primal = c0.best.dual = c0.best.gap = INFINITY;
  c0.state = kRunning;
  c0.spectral_norm = spectral_norm;
  c0.eta_ceiling = 1.0e3 / std::max(spectral_norm, 1e-12);
  c0.tolerance = prm.tolerance;
  c0.bound_norm = bound_norm;
  c0.cost_norm = cost_norm;
  c0.iteration_limit = iteration_limit;
  c0.use_restarts = prm.restart ? 1 : 0;
  c0.stop_at_request = prm.stop_at_request ? 1 : 0;
  c0.stop_rule = prm.stop_rule;
  c0.farkas_cooldown = prm.detect_infeasibility ? 0 : (1 << 30);
  if (halpern) {
    c0.halpern = 1;
    c0.eta = 0.998 / std::max(spectral_norm, 1e-12);  // constant: tau sigma ||A||^2 < 1
  }
  L64.halpern = L32.halpern = halpern;

  // the time limit counts from the start of the call, like the reference's Timer
  mark("norm estimate and A x0");
  const double setup_seconds = seconds_since(t_start);
  if (std::isfinite(prm.time_limit) && prm.time_limit > 0.0) {
    unsigned long long* d_now = a.zeros<unsigned long long>(1);
    read_clock_kernel<<<1, 1, 0, stream>>>(d_now);
    ++g_launches;
    unsigned long long now = 0;
    SIH26_CUDA(cudaMemcpyAsync(&now, d_now, sizeof now, cudaMemcpyDeviceToHost, stream),
               SANKHYA_GPU_COPY_FAILED);
    SIH26_CUDA(cudaStreamSynchronize(stream), SANKHYA_GPU_SYNC_FAILED);
    const double left = prm.time_limit - seconds_since(t_start);
    cm.bar.deadline_ns = now + static_cast<unsigned long long>(std::max(0.0, left) * 1e9);
    L64.S.bar = cm.bar;
    L32.S.bar = cm.bar;
    if (left <= 0.0) {
      int one = 1;
      SIH26_CUDA(cudaMemcpy(flags + 1, &one, sizeof one, cudaMemcpyHostToDevice), SANKHYA_GPU_COPY_FAILED);
      c0.time_up = 1;
    }
  }
  // Fault injection for the grid barrier's give-up path, for tests only: with
  // SANKHYA_PDHG_TEST_BARRIER_FAULT=<ms> in the environment the last block of the iteration
  // kernel never arrives at its first barrier, and the others give up after <ms> ms, so the
  // call must end with DEVICE_TIMEOUT and leave the context usable.
  if (const char* fault = std::getenv("SANKHYA_PDHG_TEST_BARRIER_FAULT")) {
    const double ms = std::atof(fault);
    const unsigned long long limit =
        static_cast<unsigned long long>((ms > 0.0 ? std::min(ms, 4000.0) : 200.0) * 1e6);
    L64.S.bar.skip_block = L32.S.bar.skip_block = G - 1;
    L64.S.bar.limit_ns = L32.S.bar.limit_ns = limit;
  }

  // the pinned control-block mirror: one per calling thread, kept for the thread's lifetime
  // (a pinned allocation per call costs as much as a small LP's whole setup)
  thread_local Ctrl* host_ctrl = nullptr;
  if (!host_ctrl) SIH26_CUDA(cudaMallocHost(&host_ctrl, sizeof(Ctrl)), SANKHYA_GPU_OUT_OF_MEMORY);

  cudaEvent_t ev0, ev1;
  SIH26_CUDA(cudaEventCreate(&ev0), SANKHYA_GPU_INIT_FAILED);
  SIH26_CUDA(cudaEventCreate(&ev1), SANKHYA_GPU_INIT_FAILED);
  struct EvFree {
    cudaEvent_t a, b;
    ~EvFree() { cudaEventDestroy(a); cudaEventDestroy(b); }
  } ef{ev0, ev1};

  if (prm.verbose) {
    std::printf("GPU PDHG: %d rows, %d columns, %lld nonzeros, %d blocks x %d threads, ||A||_2 ~ %.4e\n",
                m, n, q.nnz, G, kThreads, spectral_norm);
    double prev = 0.0;
    std::printf("setup:");
    for (const auto& mk : marks) {
      std::printf(" %s %.1f ms;", mk.first, (mk.second - prev) * 1e3);
      prev = mk.second;
    }
    std::printf("\n");
    std::printf("%10s %12s %10s %10s %10s %9s %9s\n", "iteration", "objective", "primal", "dual",
                "gap", "eta", "omega");
  }
  LaunchTimer timer;
  timer.on = prm.profile_kernels != 0;
  SIH26_CUDA(cudaEventRecord(ev0, stream), SANKHYA_GPU_INIT_FAILED);
  Ctrl fin{};
  Certificate cert;
  long long fp32_iterations = 0;
  if (!mixed) {
    a.put(cm.ctrl, &c0, sizeof(Ctrl), stream);
    fin = run_loop_checked(L64, G, stream, host_ctrl, prm.verbose, 0, nullptr, timer, prob, q, a,
                           cm.cert_row, cm.cert_col, cert);
  } else {
    // FP32 phase: relative KKT to the switch tolerance -- by default the request, but no
    // finer than kFp32Reach -- handing over early if the FP32 level stalls
    const double fp32_target =
        prm.mixed_switch_tolerance > 0.0 ? std::max(prm.tolerance, prm.mixed_switch_tolerance)
                                         : std::max(prm.tolerance, kFp32Reach);
    Ctrl c32 = c0;
    c32.stop_rule = 1;
    c32.tolerance = fp32_target;
    a.put(cm.ctrl, &c32, sizeof(Ctrl), stream);
    bool stalled = false;
    const int stall_checks = prm.mixed_stall_checks > 0 ? prm.mixed_stall_checks
                           : prm.mixed_stall_checks < 0 ? 0 : kAutoStall;
    fin = run_loop_checked(L32, G, stream, host_ctrl, prm.verbose, stall_checks, &stalled, timer,
                           prob, q, a, cm.cert_row, cm.cert_col, cert);
    fp32_iterations = fin.iteration;
    const bool done_in_fp32 = fin.state == kConverged && prm.stop_rule == 1 &&
                              fp32_target <= prm.tolerance;
    const bool limit_hit = fin.state == kIterationLimit || fin.state == kTimeLimit ||
                           fin.state == kDeviceError || cert.kind != 0;
    if (!done_in_fp32 && !limit_hit) {
      // FP64 polish. The hand-over keeps the whole restart state -- iterate, restart anchor,
      // running sums and their count, step size, primal weight -- so the FP64 loop goes on
      // exactly where the FP32 one stopped, only with more digits.
      const int threads = 256, blocks = std::max(1, std::min(4096, (std::max(m, n) + threads - 1) / threads));
      handover_kernel<<<blocks, threads, 0, stream>>>(L32.S, fin.cur, static_cast<double>(fin.averaged),
                                                     L64.S, m, n, halpern ? 1 : 0);
      SIH26_CUDA(cudaGetLastError(), SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
      ++g_launches;
      Ctrl h = fin;
      h.cur = 0;
      h.state = kRunning;
      h.converged = 0;
      h.tolerance = prm.tolerance;
      h.stop_rule = prm.stop_rule;
      if (halpern) {
        // the Halpern sequence restarts at the hand-over point
        h.averaged = 0;
        h.last_restart = h.iteration;
      }
      a.put(cm.ctrl, &h, sizeof(Ctrl), stream);
      init_ax_kernel<double><<<G, kThreads, stream_smem_bytes(), stream>>>(L64.P, L64.S);
      SIH26_CUDA(cudaGetLastError(), SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
      ++g_launches;
      if (halpern)
        SIH26_CUDA(cudaMemcpyAsync(L64.S.axr, L64.S.ax[0], m * sizeof(double),
                                   cudaMemcpyDeviceToDevice, stream), SANKHYA_GPU_COPY_FAILED);
      fin = run_loop_checked(L64, G, stream, host_ctrl, prm.verbose, 0, nullptr, timer, prob, q,
                             a, cm.cert_row, cm.cert_col, cert);
    }
  }
  SIH26_CUDA(cudaEventRecord(ev1, stream), SANKHYA_GPU_INIT_FAILED);
  if (fin.state == kDeviceError)
    throw Failure{SANKHYA_GPU_DEVICE_TIMEOUT, "a grid barrier timed out during the iteration loop"};

  // ---- report (pdhg.cpp:647-716) ----
  double* d_x = a.zeros<double>(n);
  double* d_red = a.zeros<double>(n);
  double* d_y = a.zeros<double>(m);
  {
    void* ra[] = {&L64.P, &L64.S, &d_x, &d_red, &d_y};
    launch_coop(reinterpret_cast<const void*>(report_kernel<double>), G, ra, stream_smem_bytes(), stream);
  }
  SIH26_CUDA(cudaMemcpyAsync(host_ctrl, cm.ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, stream),
             SANKHYA_GPU_COPY_FAILED);
  std::vector<double> hx(n), hred(n), hy(m);
  a.get(hx.data(), d_x, n * 8, stream);
  a.get(hred.data(), d_red, n * 8, stream);
  a.get(hy.data(), d_y, m * 8, stream);
  SIH26_CUDA(cudaStreamSynchronize(stream), SANKHYA_GPU_SYNC_FAILED);
  const Ctrl rep = *host_ctrl;
  if (rep.state == kDeviceError)
    throw Failure{SANKHYA_GPU_DEVICE_TIMEOUT, "a grid barrier timed out in the report"};
  float ms = 0.f;
  SIH26_CUDA(cudaEventElapsedTime(&ms, ev0, ev1), SANKHYA_GPU_SYNC_FAILED);

  // un-permute
  std::vector<double> col_value(n), reduced(n), y(m);
  for (int t = 0; t < n; ++t) {
    col_value[q.col_perm[t]] = hx[t];
    reduced[q.col_perm[t]] = hred[t];
  }
  for (int t = 0; t < m; ++t) y[q.row_perm[t]] = hy[t];
  for (double v : col_value)
    if (!std::isfinite(v)) throw Failure{SANKHYA_GPU_NON_FINITE_OUTPUT, "the reported point is not finite"};
  if (res->col_value) std::memcpy(res->col_value, col_value.data(), n * sizeof(double));
  if (res->col_dual) for (int j = 0; j < n; ++j) res->col_dual[j] = sense * reduced[j];
  if (res->row_dual) for (int i = 0; i < m; ++i) res->row_dual[i] = sense * (-y[i]);

  const Residuals& f = rep.best;
  res->residuals = sankhya_pdhg_residuals{f.primal, f.dual, f.gap, f.primal_objective,
                                          f.dual_objective, f.absolute_primal, f.absolute_dual,
                                          f.gap_as_verified, f.complementarity};
  res->iterations = fin.iteration;
  res->attempts = fin.attempts;
  res->restarts = fin.restarts;
  res->evaluations = fin.evaluations;
  res->fp32_iterations = fp32_iterations;
  res->spectral_norm = spectral_norm;
  res->converged = fin.converged;
  double obj = prob.objective_offset;  // Model::evaluate_objective (src/core/model.cpp:99-105)
  for (int j = 0; j < n; ++j) obj += prob.cost[j] * col_value[j];
  res->objective = obj;

  const bool project_standard = f.absolute_primal <= 1e-7 && f.absolute_dual <= 1e-7 &&
                                f.gap_as_verified <= 1e-9 && f.complementarity <= 1e-6;
  const bool verifiable = fin.converged && project_standard;
  char msg[512];
  if (cert.kind == kInfeasible) {
    res->status = SANKHYA_PDHG_INFEASIBLE;
    if (res->farkas_dual) std::memcpy(res->farkas_dual, cert.value.data(), m * sizeof(double));
    std::snprintf(msg, sizeof msg,
                  "primal infeasible: Farkas certificate from the dual movement after %lld "
                  "iterations (normalised margin %.3e), checked on the original model",
                  fin.iteration, fin.farkas_margin);
  } else if (cert.kind == kUnbounded) {
    res->status = SANKHYA_PDHG_UNBOUNDED;
    if (res->primal_ray) std::memcpy(res->primal_ray, cert.value.data(), n * sizeof(double));
    std::snprintf(msg, sizeof msg,
                  "unbounded: primal ray from the last step after %lld iterations, checked on "
                  "the original model",
                  fin.iteration);
  } else if (verifiable) {
    res->status = SANKHYA_PDHG_OPTIMAL;
    std::snprintf(msg, sizeof msg,
                  "converged after %lld iterations and %lld restarts; absolute primal %.3e, dual "
                  "%.3e, relative gap %.3e",
                  fin.iteration, fin.restarts, f.absolute_primal, f.absolute_dual, f.gap_as_verified);
  } else if (fin.converged) {
    res->status = SANKHYA_PDHG_FEASIBLE;
    std::snprintf(msg, sizeof msg,
                  "met the requested relative tolerance %.1e after %lld iterations, but NOT the "
                  "absolute standard this project verifies against (primal %.3e vs 1.0e-07, dual "
                  "%.3e vs 1.0e-07, relative gap %.3e vs 1.0e-09). Reported as feasible, not "
                  "optimal. %s",
                  prm.tolerance, fin.iteration, f.absolute_primal, f.absolute_dual,
                  f.gap_as_verified,
                  prm.stop_at_request ? "pdhg_stop_at_request is on, so this is the cheap answer "
                                        "that was asked for; turn it off to run on to the standard"
                                      : "Tighten --option pdhg_tolerance to close it");
  } else {
    res->status = fin.state == kTimeLimit ? SANKHYA_PDHG_TIME_LIMIT : SANKHYA_PDHG_ITERATION_LIMIT;
    std::snprintf(msg, sizeof msg,
                  "stopped at relative primal %.3e, dual %.3e, gap %.3e after %lld iterations and "
                  "%lld restarts (target %.1e)",
                  f.primal, f.dual, f.gap, fin.iteration, fin.restarts, prm.tolerance);
  }
  fill_message(res, msg);
  res->dual_bound = (verifiable && cert.kind == 0) ? sense * f.dual_objective + prob.objective_offset
                               : (prob.maximize ? INFINITY : -INFINITY);
  res->setup_seconds = setup_seconds;
  res->h2d_bytes = a.h2d_bytes;
  res->d2h_bytes = a.d2h_bytes;
  res->iterate_kernel_seconds = timer.seconds;
  res->iterate_launches = timer.launches;
  res->kernel_launches = g_launches;
  res->autotuned = autotuned;
  res->primal_infeasibility = rep.primal_violation;
  res->quality = quality_from_slots(rep.quality, res->objective, res->dual_bound);
  res->quality.primal_infeasibility = res->primal_infeasibility;  // one figure for both fields
  res->schedule[0] = sched_a.stream_row_max;
  res->schedule[1] = sched_a.nnz_per_lane;
  res->schedule[2] = sched_at.stream_row_max;
  res->schedule[3] = sched_at.nnz_per_lane;
  res->solve_seconds = ms * 1e-3;
  res->total_seconds = seconds_since(t_start);
  return SANKHYA_GPU_SUCCESS;
}

// An UNBOUNDED verdict claims two things: a feasible point, and a ray along which the
// objective improves without limit from it (the reference's solution files carry both, and its
// checker verifies the point before the ray, src/io/writer.cpp:195-216). The ray is certified;
// the point the loop stopped at is an iterate running off along the ray and need not be
// feasible. So the same constraints are solved once more with zero cost under the reference's
// stop rule: its optimum meets the absolute standard (primal residual <= 1e-7), i.e. it is a
// feasible point, and it is reported with the ray. If that solve proves the constraints
// infeasible, the verdict is INFEASIBLE with its certificate; if it ends without a feasible
// point, the verdict is INFEASIBLE_OR_UNBOUNDED: the ray alone, no point claimed.
static void start_point_for_ray(const sankhya_pdhg_problem& prob, const sankhya_pdhg_params& prm,
                                sankhya_pdhg_result* res) {
  const int m = prob.num_rows, n = prob.num_cols;
  std::vector<double> zero(n, 0.0), x(n), rd(m), cd(n), fk(m), ray(n);
  sankhya_pdhg_problem feas = prob;
  feas.cost = zero.data();
  feas.maximize = 0;
  feas.objective_offset = 0.0;
  sankhya_pdhg_params fp = prm;
  fp.tolerance = std::min(prm.tolerance, 1e-9);
  fp.stop_rule = SANKHYA_PDHG_STOP_REFERENCE;
  fp.stop_at_request = 0;
  fp.precision = SANKHYA_PDHG_FP64;
  fp.algorithm = SANKHYA_PDHG_ALGORITHM_HALPERN;
  fp.detect_infeasibility = 1;
  fp.verbose = 0;
  fp.autotune = 0;
  fp.profile_kernels = 0;
  const long long cap = prm.iteration_limit < 0 ? 1000000ll : prm.iteration_limit;
  fp.iteration_limit = std::max<long long>(1000, cap - res->iterations);
  sankhya_pdhg_result r{};
  r.col_value = x.data();
  r.row_dual = rd.data();
  r.col_dual = cd.data();
  r.farkas_dual = fk.data();
  r.primal_ray = ray.data();
  const long long launches = g_launches;
  int rc = SANKHYA_GPU_SUCCESS;
  try {
    rc = solve_impl(feas, fp, &r);
  } catch (const Failure& f) {
    rc = f.code;
  }
  g_launches += launches;
  res->kernel_launches = g_launches;
  res->iterations += r.iterations;
  res->attempts += r.attempts;
  res->total_seconds += r.total_seconds;
  res->h2d_bytes += r.h2d_bytes;
  res->d2h_bytes += r.d2h_bytes;
  char msg[512];
  if (rc == SANKHYA_GPU_SUCCESS && r.status == SANKHYA_PDHG_OPTIMAL) {
    if (res->col_value) std::memcpy(res->col_value, x.data(), n * sizeof(double));
    if (res->row_dual) std::fill(res->row_dual, res->row_dual + m, 0.0);
    if (res->col_dual) std::memcpy(res->col_dual, prob.cost, n * sizeof(double));
    double obj = prob.objective_offset;
    for (int j = 0; j < n; ++j) obj += prob.cost[j] * x[j];
    res->objective = obj;
    res->primal_infeasibility = r.primal_infeasibility;
    res->quality.primal_infeasibility = r.quality.primal_infeasibility;
    res->quality.primal_infeasibility_scaled = r.quality.primal_infeasibility_scaled;
    std::snprintf(msg, sizeof msg, "%s; the ray starts from a feasible point found by a "
                  "zero-cost solve of the constraints in %lld iterations", res->message,
                  static_cast<long long>(r.iterations));
  } else if (rc == SANKHYA_GPU_SUCCESS && r.status == SANKHYA_PDHG_INFEASIBLE) {
    res->status = SANKHYA_PDHG_INFEASIBLE;
    if (res->farkas_dual) std::memcpy(res->farkas_dual, fk.data(), m * sizeof(double));
    std::snprintf(msg, sizeof msg, "primal infeasible (a primal ray exists too): %s", r.message);
  } else {
    res->status = SANKHYA_PDHG_INFEASIBLE_OR_UNBOUNDED;
    std::snprintf(msg, sizeof msg, "%s; no feasible point was found for the ray to start from "
                  "(zero-cost solve: %s), so unboundedness is not claimed", res->message,
                  rc == SANKHYA_GPU_SUCCESS ? r.message : "failed");
  }
  fill_message(res, msg);
}

}  // namespace sih26

extern "C" {

void sankhya_pdhg_gpu_default_params(sankhya_pdhg_params* p) {
  std::memset(p, 0, sizeof *p);
  p->tolerance = 1e-4;
  p->iteration_limit = -1;
  p->time_limit = INFINITY;
  p->restart = 1;
  p->stop_at_request = 0;
  p->random_seed = 0;
  p->precision = SANKHYA_PDHG_FP64;
  p->stop_rule = SANKHYA_PDHG_STOP_REFERENCE;
  p->device = 0;
  p->verbose = 0;
  p->detect_infeasibility = 1;
  p->mixed_switch_tolerance = 0.0;
}

int sankhya_pdhg_gpu_solve(const sankhya_pdhg_problem* problem, const sankhya_pdhg_params* params,
                           sankhya_pdhg_result* result) {
  using namespace sih26;
  if (!problem || !result) {
    g_last_error = "problem and result must not be NULL";
    return SANKHYA_GPU_INVALID_ARGUMENT;
  }
  sankhya_pdhg_params defaults;
  sankhya_pdhg_gpu_default_params(&defaults);
  DeviceGuard guard;
  try {
    const sankhya_pdhg_params& prm = params ? *params : defaults;
    const int rc = solve_impl(*problem, prm, result);
    if (rc == SANKHYA_GPU_SUCCESS && result->status == SANKHYA_PDHG_UNBOUNDED)
      start_point_for_ray(*problem, prm, result);
    return rc;
  } catch (const Failure& f) {
    g_last_error = f.message;
    std::snprintf(result->message, sizeof result->message, "%s", f.message.c_str());
    result->status = SANKHYA_PDHG_NUMERICAL_ERROR;
    return f.code;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return SANKHYA_GPU_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return SANKHYA_GPU_INVALID_DEVICE_STATE;
  }
}

const char* sankhya_pdhg_gpu_last_error(void) { return sih26::g_last_error.c_str(); }

#ifdef SIH26_PHASE_TIMING
// Instrumented builds only (see SIH26_MARK in pdhg_kernels.cuh).
int sih26_phase_timing_read(unsigned long long* out, int count) {
  return cudaMemcpyFromSymbol(out, sih26::g_phase_ns, sizeof(unsigned long long) * count) ==
                 cudaSuccess ? 0 : 1;
}
int sih26_phase_timing_reset(void) {
  static unsigned long long zero[4096 * 5];
  return cudaMemcpyToSymbol(sih26::g_phase_ns, zero, sizeof zero) == cudaSuccess ? 0 : 1;
}
#endif

int sankhya_pdhg_gpu_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
  return n;
}

int sankhya_pdhg_gpu_device_name(int device, char* name, int capacity) {
  cudaDeviceProp p{};
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) {
    sih26::g_last_error = "no such device";
    return SANKHYA_GPU_NO_COMPATIBLE_DEVICE;
  }
  if (name && capacity > 0) std::snprintf(name, capacity, "%s", p.name);
  return SANKHYA_GPU_SUCCESS;
}

}  // extern "C"
