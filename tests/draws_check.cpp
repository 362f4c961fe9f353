// The library's uniform_draws (pdhg_host.cpp: mt19937 and libstdc++'s generate_canonical
// restated) against std::mt19937 with std::uniform_real_distribution<double>, the draws of the
// reference's norm estimate (src/la/scaling.cpp:168-171) and QP power iterations, compiled
// with the same standard library the reference is built with. Prints "ok" or the first
// mismatch, for tests/test_scaling_host_cpu.py.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "pdhg_host.cuh"

int main() {
  const uint32_t seeds[] = {1u, 2u, 12u, 26119u, 20260826u, 4294967295u};
  const size_t counts[] = {1, 7, 311, 312, 313, 624, 625, 5000};
  const double ranges[][2] = {{-1.0, 1.0}, {0.0, 1.0}, {-3.5, 1e3}};
  for (const uint32_t seed : seeds) {
    for (const size_t count : counts) {
      for (const auto& r : ranges) {
        std::vector<double> mine(count);
        sih26::uniform_draws(seed, r[0], r[1], count, mine.data());
        std::mt19937 rng(seed);
        std::uniform_real_distribution<double> spread(r[0], r[1]);
        for (size_t k = 0; k < count; ++k) {
          const double want = spread(rng);
          if (std::memcmp(&want, &mine[k], sizeof want) != 0) {
            std::printf("FAIL seed %u count %zu range [%g, %g] draw %zu: %.17g vs %.17g\n",
                        seed, count, r[0], r[1], k, mine[k], want);
            return 1;
          }
        }
      }
    }
  }
  std::printf("ok\n");
  return 0;
}
