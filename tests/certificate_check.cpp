// The library's own certificate checks (pdhg_host.cpp: farkas_holds, ray_holds), the ones every
// certificate passes before the library reports it, run on small LPs read from a text file.
// Each case is whitespace-separated tokens:
//   name kind(F|R|P) m n  a[m*n] (row-major, zeros not stored)  row_lower[m] row_upper[m]
//   cost[n] col_lower[n] col_upper[n]  vector (m multipliers for F, n directions for R, P)
// with "inf" / "-inf" for absent bounds. Prints "name 1" or "name 0" per case (F: farkas_holds,
// R: ray_holds), and for P, the repair of a primal-ray candidate, "name B A": B whether the
// candidate passes ray_holds as it is, A whether repair_ray succeeds and its output passes
// ray_holds. For tests/test_certificates_cpu.py.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "pdhg_host.cuh"

using namespace sih26;

static bool read_doubles(std::ifstream& in, size_t count, std::vector<double>* out) {
  out->resize(count);
  std::string tok;
  for (size_t k = 0; k < count; ++k) {
    if (!(in >> tok)) return false;
    (*out)[k] = std::strtod(tok.c_str(), nullptr);
  }
  return true;
}

int main(int argc, char** argv) {
  if (argc < 2) {
    std::printf("FAIL usage: certificate_check cases.txt\n");
    return 1;
  }
  std::ifstream in(argv[1]);
  std::string name, kind;
  int m = 0, n = 0;
  while (in >> name >> kind >> m >> n) {
    std::vector<double> dense, rl, ru, cost, cl, cu, vec;
    if (!read_doubles(in, static_cast<size_t>(m) * n, &dense) || !read_doubles(in, m, &rl) ||
        !read_doubles(in, m, &ru) || !read_doubles(in, n, &cost) || !read_doubles(in, n, &cl) ||
        !read_doubles(in, n, &cu) || !read_doubles(in, kind == "F" ? m : n, &vec)) {
      std::printf("FAIL truncated case %s\n", name.c_str());
      return 1;
    }
    std::vector<int32_t> cs{0}, ri;
    std::vector<double> val;
    for (int j = 0; j < n; ++j) {
      for (int i = 0; i < m; ++i) {
        const double a = dense[static_cast<size_t>(i) * n + j];
        if (a != 0.0) {
          ri.push_back(i);
          val.push_back(a);
        }
      }
      cs.push_back(static_cast<int32_t>(ri.size()));
    }
    sankhya_pdhg_problem p{};
    p.num_rows = m;
    p.num_cols = n;
    p.num_nonzeros = static_cast<int32_t>(ri.size());
    p.col_starts = cs.data();
    p.row_indices = ri.data();
    p.values = val.data();
    p.cost = cost.data();
    p.col_lower = cl.data();
    p.col_upper = cu.data();
    p.row_lower = rl.data();
    p.row_upper = ru.data();
    if (kind == "P") {
      const bool before = ray_holds(p, vec);
      std::vector<double> d = vec;
      const bool after = repair_ray(p, d) && ray_holds(p, d);
      std::printf("%s %d %d\n", name.c_str(), before ? 1 : 0, after ? 1 : 0);
      continue;
    }
    const bool holds = kind == "F" ? farkas_holds(p, vec) : ray_holds(p, vec);
    std::printf("%s %d\n", name.c_str(), holds ? 1 : 0);
  }
  return 0;
}
