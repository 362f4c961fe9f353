// Invariants of the host work partition (pdhg_host.cpp: partition), checked on row lengths
// read from a file: every row is owned by exactly one item or long row; the segments of a long
// row tile it in order; the per-block index arrays are monotone and end at the list sizes;
// slices hold at most 32 short rows, are padded to their longest row, and occupy disjoint
// ranges of the slice arrays; grouped items use a power-of-two lane count. Prints one summary
// line (ok or the first broken invariant) for tests/test_partition_cpu.py.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "pdhg_host.cuh"

using namespace sih26;

static int fail(const char* what, long long a = 0, long long b = 0) {
  std::printf("FAIL %s %lld %lld\n", what, a, b);
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 6) return fail("usage: lens.bin G stream_row_max nnz_per_lane sliced");
  std::FILE* f = std::fopen(argv[1], "rb");
  if (!f) return fail("cannot open lengths");
  std::vector<int> lens;
  int v = 0;
  while (std::fread(&v, 4, 1, f) == 1) lens.push_back(v);
  std::fclose(f);
  const int G = std::atoi(argv[2]);
  const Schedule sched{std::atoi(argv[3]), std::atoi(argv[4])};
  const bool sliced = std::atoi(argv[5]) != 0;
  const int rows = static_cast<int>(lens.size());
  std::vector<int> ptr(rows + 1, 0);
  for (int r = 0; r < rows; ++r) ptr[r + 1] = ptr[r] + lens[r];
  const HostPart hp = partition(ptr, G, 16, 0, sched, sliced);

  const auto monotone = [&](const std::vector<int>& b, size_t total, const char* what) {
    if (b.size() != static_cast<size_t>(G) + 1 || b[0] != 0 || b[G] != static_cast<int>(total))
      return fail(what, static_cast<long long>(b.size()), b.empty() ? -1 : b.back());
    for (int k = 0; k < G; ++k)
      if (b[k + 1] < b[k]) return fail(what, k, b[k]);
    return 0;
  };
  if (monotone(hp.blk_item_begin, hp.items.size(), "blk_item_begin")) return 1;
  if (monotone(hp.blk_seg_begin, hp.segs.size(), "blk_seg_begin")) return 1;
  if (monotone(hp.blk_long_begin, hp.longs.size(), "blk_long_begin")) return 1;

  std::vector<int> owner(rows, 0);
  long long slice_nnz = 0, slices = 0, grouped = 0;
  std::vector<std::pair<long long, long long>> ranges;
  for (const int4& it : hp.items) {
    if (it.x < 0 || it.y > rows || it.y <= it.x) return fail("item rows", it.x, it.y);
    for (int r = it.x; r < it.y; ++r) ++owner[r];
    if (it.z < 0) {
      if (!sliced) return fail("slice in an unsliced partition", it.x);
      const int n = it.y - it.x, L = -it.z;
      if (n > 32) return fail("slice rows", n);
      for (int r = it.x; r < it.y; ++r) {
        if (lens[r] > L) return fail("slice shorter than its row", r, L);
        if (lens[r] > sched.stream_row_max) return fail("long row in a slice", r, lens[r]);
        slice_nnz += lens[r];
      }
      if (it.w < 0) return fail("slice offset", it.w);
      ranges.emplace_back(it.w, static_cast<long long>(it.w) + static_cast<long long>(n) * L);
      ++slices;
    } else if (it.z > 0) {
      const int lanes = it.z;
      if (lanes > 32 || (lanes & (lanes - 1)) != 0) return fail("lane count", lanes);
      if (it.y - it.x > 32 / lanes) return fail("rows of a grouped item", it.y - it.x, lanes);
      ++grouped;
    } else if (sliced) {
      return fail("stream item in a sliced partition", it.x);
    }
  }
  for (const int4& lr : hp.longs) {
    const int r = lr.x;
    if (r < 0 || r >= rows) return fail("long row", r);
    ++owner[r];
    // its segments, in order, tile the row
    long long at = ptr[r];
    for (int q = lr.y; q < lr.y + lr.z; ++q) {
      if (q < 0 || q >= static_cast<int>(hp.segs.size())) return fail("segment index", q);
      const int4 sg = hp.segs[q];
      if (sg.x != r || sg.y != at || sg.z <= sg.y || sg.z - sg.y > 512)
        return fail("segment", r, q);
      at = sg.z;
    }
    if (at != ptr[r + 1]) return fail("segments do not cover the row", r, at);
  }
  for (int r = 0; r < rows; ++r)
    if (owner[r] != 1) return fail("row owned", r, owner[r]);
  std::sort(ranges.begin(), ranges.end());
  for (size_t k = 0; k < ranges.size(); ++k) {
    if (ranges[k].second > hp.sell_entries) return fail("slice past the arrays", k);
    if (k > 0 && ranges[k].first < ranges[k - 1].second) return fail("slices overlap", k);
  }
  std::printf("ok rows %d items %zu slices %lld grouped %lld longs %zu segs %zu sell %lld "
              "slice_nnz %lld\n",
              rows, hp.items.size(), slices, grouped, hp.longs.size(), hp.segs.size(),
              hp.sell_entries, slice_nnz);
  return 0;
}
