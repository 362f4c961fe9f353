// The library's host build_scaling (pdhg_host.cpp; src/la/scaling.cpp:111-158 restated) on an
// LP read from a binary file, its eight outputs written to another, for
// tests/test_scaling_host_cpu.py to compare bit for bit with the reference's own build_scaling.
//   input:  int32 m, n, nnz, ruiz_rounds; int32 col_starts[n+1], row_indices[nnz];
//           f64 values[nnz], min_cost[n], col_lower[n], col_upper[n], row_lower[m],
//           row_upper[m]
//   output: f64 dr[m], dc[n], values[nnz], cost[n], col_lower[n], col_upper[n],
//           row_lower[m], row_upper[m]
#include <cstdio>
#include <vector>

#include "pdhg_host.cuh"

using namespace sih26;

template <class T>
static bool get(std::FILE* f, std::vector<T>& v, size_t count) {
  v.resize(count);
  return count == 0 || std::fread(v.data(), sizeof(T), count, f) == count;
}

template <class T>
static void put(std::FILE* f, const std::vector<T>& v) {
  if (!v.empty()) std::fwrite(v.data(), sizeof(T), v.size(), f);
}

int main(int argc, char** argv) {
  if (argc < 3) {
    std::printf("FAIL usage: scaling_check in.bin out.bin\n");
    return 1;
  }
  std::FILE* in = std::fopen(argv[1], "rb");
  if (!in) {
    std::printf("FAIL cannot open input\n");
    return 1;
  }
  int32_t head[4];
  std::vector<int32_t> cs, ri;
  std::vector<double> val, cost, cl, cu, rl, ru;
  bool ok = std::fread(head, sizeof head, 1, in) == 1;
  const size_t m = ok ? head[0] : 0, n = ok ? head[1] : 0, nnz = ok ? head[2] : 0;
  ok = ok && get(in, cs, n + 1) && get(in, ri, nnz) && get(in, val, nnz) && get(in, cost, n) &&
       get(in, cl, n) && get(in, cu, n) && get(in, rl, m) && get(in, ru, m);
  std::fclose(in);
  if (!ok) {
    std::printf("FAIL truncated input\n");
    return 1;
  }
  sankhya_pdhg_problem p{};
  p.num_rows = head[0];
  p.num_cols = head[1];
  p.num_nonzeros = head[2];
  p.col_starts = cs.data();
  p.row_indices = ri.data();
  p.values = val.data();
  p.cost = cost.data();
  p.col_lower = cl.data();
  p.col_upper = cu.data();
  p.row_lower = rl.data();
  p.row_upper = ru.data();
  const Scaling s = build_scaling(p, cost, head[3]);
  std::FILE* out = std::fopen(argv[2], "wb");
  if (!out) {
    std::printf("FAIL cannot open output\n");
    return 1;
  }
  put(out, s.dr);
  put(out, s.dc);
  put(out, s.values);
  put(out, s.cost);
  put(out, s.cl);
  put(out, s.cu);
  put(out, s.rl);
  put(out, s.ru);
  std::fclose(out);
  std::printf("ok\n");
  return 0;
}
