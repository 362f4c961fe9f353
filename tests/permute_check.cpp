// The library's host permute (pdhg_host.cpp): rows of A and of A' sorted by nonzero count,
// longest first (stable), with CSR copies in that order whose column indices point into the
// other permuted space. Reads an LP (the binary layout of tests/scaling_check.cpp, ruiz field
// ignored), permutes its values as given, and writes the outputs for
// tests/test_scaling_host_cpu.py to check against the CSC:
//   int32 row_perm[m], col_perm[n], a_ptr[m+1], a_idx[nnz], at_ptr[n+1], at_idx[nnz];
//   f64 a_val[nnz], at_val[nnz]
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
    std::printf("FAIL usage: permute_check in.bin out.bin\n");
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
  const PermutedLp q = permute(p, val);
  std::FILE* out = std::fopen(argv[2], "wb");
  if (!out) {
    std::printf("FAIL cannot open output\n");
    return 1;
  }
  put(out, q.row_perm);
  put(out, q.col_perm);
  put(out, q.a_ptr);
  put(out, q.a_idx);
  put(out, q.at_ptr);
  put(out, q.at_idx);
  put(out, q.a_val);
  put(out, q.at_val);
  std::fclose(out);
  std::printf("ok\n");
  return 0;
}
