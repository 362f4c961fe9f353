// KKT residuals of a given point for an LP already in device memory, computed without
// allocating anything (sankhya_pdhg_gpu_residuals_noalloc in include/sankhya_pdhg_gpu.h).
//
// Who needs this: a caller that must not allocate device memory once it is running -- an
// application whose device memory is owned by its own pool or arena and forbids raw
// cudaMalloc/cudaFree, a service that fixes its device-memory budget at start-up, or a
// latency-critical loop where cudaMalloc/cudaFree's implicit device synchronisation is not
// acceptable. Such a caller still wants to check an answer on the device, with the same
// residual definitions the solver uses.
//
// All scratch lives in one file-scope device array, g_noalloc_scratch, of fixed size
// (kScratchDoubles doubles = 4 MiB). Every GPU that loads this library holds it until the
// process exits. Its layout: block partials of the two reduction passes, an error word, then
// one FP64 activity slot per row, so a call accepts at most kMaxRows rows.
//
// Every call uses the same array and leaves its contents behind; each call clears what must
// start at zero (the activity accumulators and the error word) before using it. Calls whose
// work overlaps on the GPU (different streams, or different host threads without ordering)
// race on the array and give wrong answers; order them on one stream.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <string>

#include "sankhya_pdhg_gpu.h"

namespace sih26 {
extern thread_local std::string g_last_error;
}

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 512;
constexpr int kSlots = 8;
constexpr size_t kScratchDoubles = (size_t)1 << 19;  // 4 MiB
constexpr size_t kPartialDoubles = 2 * (size_t)kMaxBlocks * kSlots;
constexpr size_t kErrorDoubles = 32;  // one 256-byte line for the error word
constexpr size_t kMaxRows = kScratchDoubles - kPartialDoubles - kErrorDoubles;
static_assert(kMaxRows == SANKHYA_PDHG_NOALLOC_MAX_ROWS, "header and scratch layout disagree");

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

struct View {
  double* col_partials;  // [kMaxBlocks][kSlots]
  double* row_partials;  // [kMaxBlocks][kSlots]
  unsigned* error;       // nonzero: an index was out of range
  double* activity;      // [m]
};

__host__ __device__ inline View carve(double* base) {
  View v;
  v.col_partials = base;
  v.row_partials = base + (size_t)kMaxBlocks * kSlots;
  v.error = reinterpret_cast<unsigned*>(base + kPartialDoubles);
  v.activity = base + kPartialDoubles + kErrorDoubles;
  return v;
}

// An absent bound is +-inf or |v| >= 1e30; anything else, NaN included, is a finite bound, as
// is_finite_bound (include/sankhya/types.hpp:32-39) decides.
__device__ inline bool finite_bound(double v) { return !(fabs(v) >= 1e30); }
__device__ inline double dmax(double a, double b) { return (a < b) ? b : a; }
__device__ inline double dmin(double a, double b) { return (b < a) ? b : a; }

template <int NS>
__device__ inline void block_sum_write(double (&v)[NS], unsigned max_mask, double* out) {
  __shared__ double sh[kThreads / 32][NS];
  for (int off = 16; off > 0; off >>= 1) {
    for (int s = 0; s < NS; ++s) {
      const double o = __shfl_xor_sync(0xffffffffu, v[s], off);
      v[s] = ((max_mask >> s) & 1u) ? dmax(v[s], o) : v[s] + o;
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0)
    for (int s = 0; s < NS; ++s) sh[warp][s] = v[s];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < NS; ++s) {
      double t = sh[0][s];
      for (int w = 1; w < kThreads / 32; ++w)
        t = ((max_mask >> s) & 1u) ? dmax(t, sh[w][s]) : t + sh[w][s];
      out[(size_t)blockIdx.x * kSlots + s] = t;
    }
  }
}

__global__ void clear_kernel(double* base, int m) {
  const View v = carve(base);
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride) v.activity[i] = 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) *v.error = 0u;
}

// Columns: scatter A x into the activity slots; reduced cost d = c + A'y with the column
// terms of the reference's evaluate() (src/pdhg/pdhg.cpp:172-199, 239-256).
// slots: 0 dual violation^2, 1 bound contribution, 2 complementarity (max), 3 c'x, 4 ||c||^2
__global__ void __launch_bounds__(kThreads) column_kernel(sankhya_pdhg_problem p, const double* x,
                                                          const double* row_dual, double* base) {
  const View v = carve(base);
  const double sense = p.maximize ? -1.0 : 1.0;
  double acc[kSlots] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int stride = gridDim.x * blockDim.x;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p.num_cols; j += stride) {
    int kb = p.col_starts[j], ke = p.col_starts[j + 1];
    kb = kb < 0 ? 0 : (kb > p.num_nonzeros ? p.num_nonzeros : kb);
    ke = ke < kb ? kb : (ke > p.num_nonzeros ? p.num_nonzeros : ke);
    const double xj = x[j];
    const double c = sense * p.cost[j];
    double d = c;
    for (int k = kb; k < ke; ++k) {
      const int i = p.row_indices[k];
      if ((unsigned)i >= (unsigned)p.num_rows) {
        atomicOr(v.error, 1u);
        continue;
      }
      atomicAdd(v.activity + i, p.values[k] * xj);
      d += p.values[k] * (-sense * row_dual[i]);  // y = -sense * row_dual (pdhg.cpp:660)
    }
    const double lo = p.col_lower[j], hi = p.col_upper[j];
    if (d > 0.0) {
      if (finite_bound(lo)) acc[1] += d * lo; else acc[0] += d * d;
    } else if (d < 0.0) {
      if (finite_bound(hi)) acc[1] += d * hi; else acc[0] += d * d;
    }
    if (lo != hi) {
      const double ls = finite_bound(lo) ? xj - lo : INFINITY;
      const double us = finite_bound(hi) ? hi - xj : INFINITY;
      acc[2] = dmax(acc[2], fabs(d) * dmin(ls, us));
    }
    acc[3] += c * xj;
    acc[4] += c * c;
  }
  block_sum_write<kSlots>(acc, 1u << 2, v.col_partials);
}

// Rows (pdhg.cpp:152-170, 205-222, 227-238). slots: 0 primal violation^2, 1 support,
// 2 row dual violation^2, 3 complementarity (max), 4 ||b||^2
__global__ void __launch_bounds__(kThreads) row_kernel(sankhya_pdhg_problem p, const double* row_dual,
                                                       double* base) {
  const View v = carve(base);
  const double sense = p.maximize ? -1.0 : 1.0;
  double acc[kSlots] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < p.num_rows; i += stride) {
    const double a = v.activity[i];
    const double lo = p.row_lower[i], hi = p.row_upper[i];
    const double y = -sense * row_dual[i];
    double viol = 0.0;
    if (finite_bound(lo)) viol = dmax(viol, lo - a);
    if (finite_bound(hi)) viol = dmax(viol, a - hi);
    acc[0] += viol * viol;
    if (y > 0.0) {
      if (finite_bound(hi)) acc[1] += y * hi; else acc[2] += y * y;
    } else if (y < 0.0) {
      if (finite_bound(lo)) acc[1] += y * lo; else acc[2] += y * y;
    }
    if (lo != hi) {
      const double ls = finite_bound(lo) ? a - lo : INFINITY;
      const double us = finite_bound(hi) ? hi - a : INFINITY;
      acc[3] = dmax(acc[3], fabs(y) * dmin(ls, us));
    }
    const double b = finite_bound(lo) ? lo : (finite_bound(hi) ? hi : 0.0);
    acc[4] += b * b;
  }
  block_sum_write<kSlots>(acc, 1u << 3, v.row_partials);
}

// One thread folds the block partials in block order and writes the residual block in the
// order of sankhya_pdhg_residuals (NaN everywhere when an index was out of range).
__global__ void finish_kernel(double* base, int col_blocks, int row_blocks, double* out) {
  const View v = carve(base);
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double c[kSlots] = {0, 0, 0, 0, 0, 0, 0, 0}, r[kSlots] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = 0; b < col_blocks; ++b)
    for (int s = 0; s < kSlots; ++s) {
      const double t = v.col_partials[(size_t)b * kSlots + s];
      c[s] = s == 2 ? dmax(c[s], t) : c[s] + t;
    }
  for (int b = 0; b < row_blocks; ++b)
    for (int s = 0; s < kSlots; ++s) {
      const double t = v.row_partials[(size_t)b * kSlots + s];
      r[s] = s == 3 ? dmax(r[s], t) : r[s] + t;
    }
  if (*v.error != 0u) {
    for (int k = 0; k < 9; ++k) out[k] = NAN;
    return;
  }
  const double bound_norm = sqrt(r[4]), cost_norm = sqrt(c[4]);
  const double abs_primal = sqrt(r[0]);
  const double abs_dual = sqrt(c[0] + r[2]);
  const double pobj = c[3], dobj = c[1] - r[1];
  const double gap = fabs(pobj - dobj);
  out[0] = abs_primal / (1.0 + bound_norm);
  out[1] = abs_dual / (1.0 + cost_norm);
  out[2] = gap / (1.0 + fabs(pobj) + fabs(dobj));
  out[3] = pobj;
  out[4] = dobj;
  out[5] = abs_primal;
  out[6] = abs_dual;
  out[7] = gap / dmax(1.0, fabs(pobj));
  out[8] = dmax(c[2], r[3]);
}

// Device address of g_noalloc_scratch on the current device. In host code the array's name is
// only a stand-in for the symbol; kernels must be handed this address. It is resolved on every
// call with the caller's device current: the lookup allocates nothing and queues no work, and
// a cached address would go stale when the module is loaded again (after cudaDeviceReset, or
// under another context the caller makes current). The first call on a device is the one that
// loads this library's device code there (CUDA loads modules lazily), so make it before any
// stream capture.
int scratch_for_current_device(double** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    sih26::g_last_error = "no current CUDA device";
    return SANKHYA_GPU_NO_COMPATIBLE_DEVICE;
  }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || p == nullptr) {
    sih26::g_last_error = std::string("cudaGetSymbolAddress(g_noalloc_scratch) on device ") +
                          std::to_string(dev) + ": " + cudaGetErrorString(e);
    return SANKHYA_GPU_INIT_FAILED;
  }
  *out = static_cast<double*>(p);
  return SANKHYA_GPU_SUCCESS;
}

}  // namespace

extern "C" int sankhya_pdhg_gpu_residuals_noalloc(const sankhya_pdhg_problem* problem,
                                                  const double* x, const double* row_dual,
                                                  double* residuals_out, void* stream) {
  using sih26::g_last_error;
  if (!problem || !x || !residuals_out || (problem->num_rows > 0 && !row_dual)) {
    g_last_error = "problem, x, row_dual and residuals_out must be device pointers, not NULL";
    return SANKHYA_GPU_INVALID_ARGUMENT;
  }
  const sankhya_pdhg_problem& p = *problem;
  if (p.num_rows < 0 || p.num_cols < 0 || p.num_nonzeros < 0 || !p.col_starts ||
      (p.num_nonzeros > 0 && (!p.row_indices || !p.values)) ||
      (p.num_cols > 0 && (!p.cost || !p.col_lower || !p.col_upper)) ||
      (p.num_rows > 0 && (!p.row_lower || !p.row_upper))) {
    g_last_error = "malformed problem: negative size or NULL array";
    return SANKHYA_GPU_INVALID_ARGUMENT;
  }
  if ((size_t)p.num_rows > kMaxRows) {
    char buf[160];
    std::snprintf(buf, sizeof buf,
                  "%d rows exceed the %zu this entry point's fixed scratch can hold; use "
                  "sankhya_pdhg_gpu_solve, which allocates",
                  p.num_rows, kMaxRows);
    g_last_error = buf;
    return SANKHYA_GPU_INVALID_ARGUMENT;
  }
  double* base = nullptr;
  const int rc = scratch_for_current_device(&base);
  if (rc != SANKHYA_GPU_SUCCESS) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const auto blocks_for = [](int count) {
    int b = (count + kThreads - 1) / kThreads;
    return b < 1 ? 1 : (b > kMaxBlocks ? kMaxBlocks : b);
  };
  const int cb = blocks_for(p.num_cols), rb = blocks_for(p.num_rows);
  clear_kernel<<<blocks_for(p.num_rows), kThreads, 0, s>>>(base, p.num_rows);
  column_kernel<<<cb, kThreads, 0, s>>>(p, x, row_dual, base);
  row_kernel<<<rb, kThreads, 0, s>>>(p, row_dual, base);
  finish_kernel<<<1, 32, 0, s>>>(base, cb, rb, residuals_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_last_error = std::string("launch failed: ") + cudaGetErrorString(e);
    return SANKHYA_GPU_KERNEL_LAUNCH_FAILED;
  }
  return SANKHYA_GPU_SUCCESS;
}
