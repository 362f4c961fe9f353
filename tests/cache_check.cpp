// The autotuner's cache file (pdhg_host.cpp: autotune_store / autotune_lookup, chunk_store /
// chunk_lookup, chunk_key) exercised on the CPU in a scratch directory: the directory chain
// is created, the last line of a key wins, keys match whole (not by prefix), and lines that
// are malformed, hold non-positive values or overrun the line buffer are ignored, so an
// edited or damaged cache can only fall back to measuring again. Prints "ok" or the first
// failed step, for tests/test_cache_cpu.py.
#include <cstdio>
#include <string>
#include <vector>

#include "pdhg_host.cuh"

using namespace sih26;

static int fail(const char* step) {
  std::printf("FAIL %s\n", step);
  return 1;
}

static bool same(const Schedule& x, int a, int b) {
  return x.stream_row_max == a && x.nnz_per_lane == b;
}

int main(int argc, char** argv) {
  if (argc < 2) return fail("usage: cache_check scratch_dir");
  const std::string path = std::string(argv[1]) + "/a/b/c/autotune.tsv";
  Schedule a, at;
  if (autotune_lookup(path, "k1", &a, &at)) return fail("lookup in a missing file");
  autotune_store(path, "k1", Schedule{32, 16}, Schedule{24, 8}, 10.0, 11.0);
  if (!autotune_lookup(path, "k1", &a, &at) || !same(a, 32, 16) || !same(at, 24, 8))
    return fail("store then lookup (directories created)");
  autotune_store(path, "k1", Schedule{16, 4}, Schedule{8, 2}, 9.0, 9.5);
  autotune_store(path, "k10", Schedule{4, 4}, Schedule{4, 4}, 1.0, 1.0);
  if (!autotune_lookup(path, "k1", &a, &at) || !same(a, 16, 4) || !same(at, 8, 2))
    return fail("the last line of a key wins; a longer key is another key");
  if (autotune_lookup(path, "k", &a, &at)) return fail("a prefix is not a key");
  {
    std::FILE* f = std::fopen(path.c_str(), "a");
    if (!f) return fail("append");
    std::fprintf(f, "k2\tabc\n");
    std::fprintf(f, "k2\t0\t16\t32\t16\t1\t1\n");
    std::fprintf(f, "k2\t32\t-1\t32\t16\t1\t1\n");
    std::fprintf(f, "k2 without a tab\n");
    std::fprintf(f, "%s\n", std::string(3000, 'x').c_str());
    std::fprintf(f, "k1\t7\n");  // too few fields: k1 keeps its last good line
    std::fclose(f);
  }
  if (autotune_lookup(path, "k2", &a, &at)) return fail("malformed or non-positive lines");
  if (!autotune_lookup(path, "k1", &a, &at) || !same(a, 16, 4) || !same(at, 8, 2))
    return fail("a bad line does not replace a good one");

  const std::string cpath = std::string(argv[1]) + "/d/chunks.tsv";
  long long chunk = -1;
  if (chunk_lookup(cpath, "f", &chunk)) return fail("chunk lookup in a missing file");
  chunk_store(cpath, "f", 512, 60.0);
  chunk_store(cpath, "f", 1024, 64.0);
  chunk_store(cpath, "g", 0, 1.0);
  if (!chunk_lookup(cpath, "f", &chunk) || chunk != 1024) return fail("chunk: last line wins");
  if (chunk_lookup(cpath, "g", &chunk)) return fail("chunk: zero is not a chunk");

  const std::vector<long long> nnz = {100, 5000, 2000, 70000, 300};
  const std::vector<double> per_row = {2.5, 7.0, 10.0, 4.0, 6.0};
  const std::string k1 = chunk_key(148, 1024, nnz, per_row);
  const std::string k2 = chunk_key(148, 1024, {300, 70000, 2000, 5000, 100},
                                   {6.0, 4.0, 10.0, 7.0, 2.5});
  if (k1 != k2) return fail("chunk key: the sample's order does not matter");
  if (chunk_key(132, 1024, nnz, per_row) == k1) return fail("chunk key: the SM count matters");
  if (chunk_key(148, 512, nnz, per_row) == k1) return fail("chunk key: the slots matter");
  std::printf("ok\n");
  return 0;
}
