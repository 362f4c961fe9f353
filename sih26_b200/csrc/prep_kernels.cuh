// Preparation of one LP on the device: diagonal scaling and the permuted CSR copies of A and
// A', the device twin of build_scaling / permute in pdhg_host.cpp.
//
// build_scaling (src/la/scaling.cpp:111-158): 10 Ruiz rounds (1/sqrt(max |a|) per row and
// column) and one Pock-Chambolle round (1/sqrt(sum |a|)), each applied to the values as
// v * row_pass * column_pass. Every result is bit-identical to the host code and so to the
// reference: maxima are exact; each column sum runs down its column in row order and each row
// sum along its row in column order -- the order the reference accumulates in -- one thread
// per row or column; 1/sqrt is IEEE-rounded division of an IEEE-rounded square root; products
// are plain multiplies (no fused add to contract).
//
// permute: rows of A and of A' sorted by nonzero count, longest first, ties by index (a stable
// radix sort of inverted counts), and each permuted row's entries in ascending permuted index
// (a radix sort of (row position, column position) keys).
#pragma once

#include <cstdint>

#include "device_common.cuh"

namespace sih26 {
namespace prep {

__device__ __forceinline__ long long gtid() {
  return static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
}
__device__ __forceinline__ long long gstride() {
  return static_cast<long long>(gridDim.x) * blockDim.x;
}

// col[k] = the column of CSC entry k
__global__ void column_of_entry(const int* cs, int n, int* col) {
  for (long long j = gtid(); j < n; j += gstride())
    for (int k = cs[j]; k < cs[j + 1]; ++k) col[k] = static_cast<int>(j);
}

// idx[k] = k
__global__ void identity(int* idx, long long len) {
  for (long long k = gtid(); k < len; k += gstride()) idx[k] = static_cast<int>(k);
}

// dst[i] = value
__global__ void fill(double* dst, long long len, double value) {
  for (long long k = gtid(); k < len; k += gstride()) dst[k] = value;
}

// counts[idx[k]] += 1
__global__ void count_by(const int* idx, long long len, int* counts) {
  for (long long k = gtid(); k < len; k += gstride()) atomicAdd(counts + idx[k], 1);
}

// dst[t] = src[perm[t]]
template <class T>
__global__ void gather(const int* perm, const T* src, long long len, T* dst) {
  for (long long t = gtid(); t < len; t += gstride()) dst[t] = src[perm[t]];
}

// row[t] = the row of row-major entry t
__global__ void row_of_entry(const int* rptr, int m, int* row) {
  for (long long i = gtid(); i < m; i += gstride())
    for (int t = rptr[i]; t < rptr[i + 1]; ++t) row[t] = static_cast<int>(i);
}

// out[s] = max or sum of |v| over segment s = [ptr[s], ptr[s+1]), in segment order
__global__ void segment_norms(const int* ptr, const double* v, int segments, int sum, double* out) {
  for (long long s = gtid(); s < segments; s += gstride()) {
    double acc = 0.0;
    for (int k = ptr[s]; k < ptr[s + 1]; ++k) {
      const double mag = fabs(v[k]);
      acc = sum ? acc + mag : (acc < mag ? mag : acc);
    }
    out[s] = acc;
  }
}

// p = 1/sqrt(a) where a > 0, else 1; d *= p (the accumulated scaling)
__global__ void pass_factors(const double* a, int len, double* p, double* d) {
  for (long long i = gtid(); i < len; i += gstride()) {
    const double f = a[i] > 0.0 ? 1.0 / sqrt(a[i]) : 1.0;
    p[i] = f;
    d[i] *= f;
  }
}

// v[k] = v[k] * rp[row[k]] * cp[col[k]]
__global__ void apply_pass(const int* row, const int* col, const double* rp, const double* cp,
                           long long len, double* v) {
  for (long long k = gtid(); k < len; k += gstride()) v[k] = v[k] * rp[row[k]] * cp[col[k]];
}

// scaled column vectors (scaling.cpp:124-145): cost dc, bounds times 1/dc
__global__ void scaled_columns(const double* cmin, const double* cl, const double* cu,
                               const double* dc, int n, double* c_s, double* cl_s, double* cu_s) {
  for (long long j = gtid(); j < n; j += gstride()) {
    const double d = dc[j];
    c_s[j] = cmin[j] * d;
    cl_s[j] = finite_bound(cl[j]) ? cl[j] * (1.0 / d) : cl[j];
    cu_s[j] = finite_bound(cu[j]) ? cu[j] * (1.0 / d) : cu[j];
  }
}

__global__ void scaled_rows(const double* rl, const double* ru, const double* dr, int m,
                            double* rl_s, double* ru_s) {
  for (long long i = gtid(); i < m; i += gstride()) {
    const double d = dr[i];
    rl_s[i] = finite_bound(rl[i]) ? rl[i] * d : rl[i];
    ru_s[i] = finite_bound(ru[i]) ? ru[i] * d : ru[i];
  }
}

// keys that sort segments longest first, ties by index under a stable sort: ~count
__global__ void count_keys(const int* ptr, int len, unsigned* key, int* index) {
  for (long long i = gtid(); i < len; i += gstride()) {
    key[i] = ~static_cast<unsigned>(ptr[i + 1] - ptr[i]);
    index[i] = static_cast<int>(i);
  }
}

// pos[perm[t]] = t
__global__ void positions(const int* perm, int len, int* pos) {
  for (long long t = gtid(); t < len; t += gstride()) pos[perm[t]] = static_cast<int>(t);
}

// lengths in permuted order, for the permuted row pointers
__global__ void permuted_lengths(const int* ptr, const int* perm, int len, int* out) {
  for (long long t = gtid(); t < len; t += gstride()) out[t] = ptr[perm[t] + 1] - ptr[perm[t]];
}

// (outer position << shift | inner position) for every entry; shift covers the inner positions
__global__ void pair_keys(const int* outer, const int* inner, const int* outer_pos,
                          const int* inner_pos, long long len, int shift, unsigned long long* key) {
  for (long long k = gtid(); k < len; k += gstride())
    key[k] = (static_cast<unsigned long long>(outer_pos[outer[k]]) << shift) |
             static_cast<unsigned long long>(inner_pos[inner[k]]);
}

__global__ void low_bits(const unsigned long long* key, long long len, int shift, int* idx) {
  const unsigned long long mask = (1ull << shift) - 1ull;
  for (long long k = gtid(); k < len; k += gstride()) idx[k] = static_cast<int>(key[k] & mask);
}

// the starting point (pdhg.cpp:329-334): the projection of zero onto the scaled box
__global__ void start_point(const double* cl_s, const double* cu_s, int n, double* x0) {
  for (long long j = gtid(); j < n; j += gstride()) {
    double v = 0.0;
    if (finite_bound(cl_s[j]) && v < cl_s[j]) v = cl_s[j];
    else if (finite_bound(cu_s[j]) && v > cu_s[j]) v = cu_s[j];
    x0[j] = v;
  }
}

__global__ void to_float(const double* src, long long len, float* dst) {
  for (long long k = gtid(); k < len; k += gstride()) dst[k] = static_cast<float>(src[k]);
}

}  // namespace prep
}  // namespace sih26
