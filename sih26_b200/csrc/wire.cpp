// The request wire format of include/sankhya_pdhg_gpu.h: one LP as a flat little-endian buffer
// whose arrays are 8-byte aligned, so a received request is solved in place.
#include <cstring>
#include <string>

#include "pdhg_host.cuh"
#include "sankhya_pdhg_gpu.h"

namespace sih26 {

extern thread_local std::string g_last_error;

namespace {

constexpr size_t kHeader = 32;

size_t align8(size_t v) { return (v + 7) & ~size_t(7); }

struct Offsets {
  size_t cs, ri, val, cost, cl, cu, rl, ru, end;
};

Offsets offsets(long long m, long long n, long long nnz) {
  Offsets o{};
  size_t at = kHeader;
  const auto take = [&](size_t bytes) {
    const size_t here = at;
    at = align8(at + bytes);
    return here;
  };
  o.cs = take((n + 1) * 4);
  o.ri = take(nnz * 4);
  o.val = take(nnz * 8);
  o.cost = take(n * 8);
  o.cl = take(n * 8);
  o.cu = take(n * 8);
  o.rl = take(m * 8);
  o.ru = take(m * 8);
  o.end = at;
  return o;
}

int fail(const std::string& why) {
  g_last_error = why;
  return SANKHYA_GPU_INVALID_ARGUMENT;
}

}  // namespace
}  // namespace sih26

extern "C" {

size_t sankhya_pdhg_wire_size(const sankhya_pdhg_problem* p) {
  if (!p || p->num_rows < 0 || p->num_cols < 0 || p->num_nonzeros < 0) return 0;
  return sih26::offsets(p->num_rows, p->num_cols, p->num_nonzeros).end;
}

int sankhya_pdhg_wire_write(const sankhya_pdhg_problem* p, void* buffer, size_t bytes) {
  using namespace sih26;
  if (!p || !buffer) return fail("problem and buffer must not be NULL");
  try {
    check_structure(*p);
  } catch (const Failure& f) {
    return fail(f.message);
  }
  const long long m = p->num_rows, n = p->num_cols, nnz = p->num_nonzeros;
  const Offsets o = offsets(m, n, nnz);
  if (bytes < o.end) return fail("the buffer is smaller than sankhya_pdhg_wire_size()");
  unsigned char* b = static_cast<unsigned char*>(buffer);
  std::memset(b, 0, o.end);
  std::memcpy(b, SANKHYA_PDHG_WIRE_MAGIC, 8);
  const int32_t head[4] = {p->num_rows, p->num_cols, p->num_nonzeros, p->maximize ? 1 : 0};
  std::memcpy(b + 8, head, sizeof head);
  std::memcpy(b + 24, &p->objective_offset, 8);
  std::memcpy(b + o.cs, p->col_starts, (n + 1) * 4);
  if (nnz) {
    std::memcpy(b + o.ri, p->row_indices, nnz * 4);
    std::memcpy(b + o.val, p->values, nnz * 8);
  }
  if (n) {
    std::memcpy(b + o.cost, p->cost, n * 8);
    std::memcpy(b + o.cl, p->col_lower, n * 8);
    std::memcpy(b + o.cu, p->col_upper, n * 8);
  }
  if (m) {
    std::memcpy(b + o.rl, p->row_lower, m * 8);
    std::memcpy(b + o.ru, p->row_upper, m * 8);
  }
  return SANKHYA_GPU_SUCCESS;
}

int sankhya_pdhg_wire_view(const void* buffer, size_t bytes, sankhya_pdhg_problem* p) {
  using namespace sih26;
  if (!buffer || !p) return fail("buffer and problem must not be NULL");
  if (reinterpret_cast<uintptr_t>(buffer) % 8 != 0) return fail("the buffer is not 8-byte aligned");
  if (bytes < kHeader) return fail("the buffer is shorter than the wire header");
  const unsigned char* b = static_cast<const unsigned char*>(buffer);
  if (std::memcmp(b, SANKHYA_PDHG_WIRE_MAGIC, 8) != 0) return fail("not a wire buffer (bad magic)");
  int32_t head[4];
  std::memcpy(head, b + 8, sizeof head);
  if (head[0] < 0 || head[1] < 0 || head[2] < 0) return fail("negative size in the wire header");
  const Offsets o = offsets(head[0], head[1], head[2]);
  if (bytes < o.end) return fail("the wire buffer is truncated");
  sankhya_pdhg_problem q{};
  q.num_rows = head[0];
  q.num_cols = head[1];
  q.num_nonzeros = head[2];
  q.maximize = (head[3] & 1) ? 1 : 0;
  std::memcpy(&q.objective_offset, b + 24, 8);
  q.col_starts = reinterpret_cast<const int32_t*>(b + o.cs);
  q.row_indices = reinterpret_cast<const int32_t*>(b + o.ri);
  q.values = reinterpret_cast<const double*>(b + o.val);
  q.cost = reinterpret_cast<const double*>(b + o.cost);
  q.col_lower = reinterpret_cast<const double*>(b + o.cl);
  q.col_upper = reinterpret_cast<const double*>(b + o.cu);
  q.row_lower = reinterpret_cast<const double*>(b + o.rl);
  q.row_upper = reinterpret_cast<const double*>(b + o.ru);
  try {
    check_structure(q);
  } catch (const Failure& f) {
    return fail(f.message);
  }
  *p = q;
  return SANKHYA_GPU_SUCCESS;
}

}  // extern "C"
