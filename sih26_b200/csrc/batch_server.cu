// Batched and served restarted PDHG behind the C ABI (sankhya_pdhg_server_* and
// sankhya_pdhg_gpu_batch_solve in include/sankhya_pdhg_gpu.h).
//
// A server owns one device memory pool (a fraction of free HBM, taken once at creation),
// a table of LP slots and one CUDA graph. submit() prepares an LP on the host (validation,
// scaling, permutation, work partition for one block -- or for an 8-block cluster when the
// LP has at least cluster_min_nnz nonzeros) into one contiguous device image; step() admits
// waiting LPs whose image fits the pool, replays the graph (the single-block and the cluster
// persistent kernels side by side on two forked streams, over every active LP of their
// class, each LP for at most chunk_attempts attempts),
// reads the compact control blocks back, re-checks every Farkas certificate on the host, and
// retires finished LPs with their answers. LPs admitted while others run simply join the
// next launch: that is continuous batching.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "batch_kernels.cuh"
#include "pdhg_host.cuh"
#include "sankhya_pdhg_gpu.h"

namespace sih26 {

extern thread_local std::string g_last_error;

#define SIH26_SCUDA(expr, code)                                                          \
  do {                                                                                   \
    const cudaError_t e_ = (expr);                                                       \
    if (e_ != cudaSuccess)                                                               \
      throw Failure{code, std::string(#expr) + ": " + cudaGetErrorString(e_)};           \
  } while (0)

namespace {

using Clock = std::chrono::steady_clock;

// Offsets of one LP's arrays inside its device image (bytes, 256-byte aligned).
struct Layout {
  size_t bytes = 0;
  size_t put(size_t n) {
    const size_t at = bytes;
    bytes += (n + 255) & ~size_t(255);
    return at;
  }
};

struct PartOff {
  size_t blk_seg_begin, segs, blk_long_begin, longs, blk_item_begin, items, seg_sum;
};

// One submitted LP.
struct Job {
  int64_t ticket = 0;
  int m = 0, n = 0;
  long long nnz = 0;
  // the original problem, kept for the objective, the certificate check and the outputs
  std::vector<int> cs, ri;
  std::vector<double> val, cost, cl, cu, rl, ru;
  sankhya_pdhg_problem view{};
  sankhya_pdhg_params prm{};
  std::vector<int> row_perm, col_perm;
  // the device image and where each array sits in it
  std::vector<unsigned char> image;
  struct {
    size_t a_ptr, a_idx, a_val, at_ptr, at_idx, at_val;
    PartOff pa, pat;
    size_t c, cl, cu, rl, ru, dr, dc, c0, cl0, cu0, rl0, ru0;
    size_t x0, x1, y0, y1, ax0, ax1, xsum, ysum, xr, yr, xavg, yavg, best_x, best_y;
    size_t xt, yt, axr;  // the Halpern operator's T(z) and A x_0
    size_t x_out, red_out, y_out, farkas_out, ray_out;
  } off{};
  Ctrl ctrl0{};
  // lifecycle
  int group = 1;  // blocks working on this LP: 1, or kClusterSize
  int slot = -1;
  size_t pool_offset = 0;
  size_t pool_bytes = 0;
  bool finished = false;
  bool model_error = false;
  std::string message;
  double submit_time = 0.0, admit_time = 0.0, finish_time = 0.0;
  // solved alone on the whole GPU by the single-LP engine; its result as that engine filled it
  bool solo = false;
  sankhya_pdhg_result solo_result{};
  // result
  int status = SANKHYA_PDHG_NOT_SOLVED;
  Ctrl last{};
  std::vector<double> x, row_dual, col_dual, farkas, ray;
};

template <class T>
void write(std::vector<unsigned char>& img, size_t at, const std::vector<T>& v) {
  if (!v.empty()) std::memcpy(img.data() + at, v.data(), v.size() * sizeof(T));
}

template <class T>
std::vector<T> gathered(const std::vector<T>& v, const std::vector<int>& perm) {
  std::vector<T> out(perm.size());
  for (size_t t = 0; t < perm.size(); ++t) out[t] = v[perm[t]];
  return out;
}

// Host preparation of one LP (the setup half of the single-LP solve, with G = 1).
void prepare(Job& J, const sankhya_pdhg_problem& p, const sankhya_pdhg_params& prm,
             long long cluster_min_nnz, long long solo_min_nnz) {
  check_structure(p);
  const int m = p.num_rows, n = p.num_cols;
  J.m = m;
  J.n = n;
  J.nnz = p.num_nonzeros;
  J.prm = prm;
  J.cs.assign(p.col_starts, p.col_starts + n + 1);
  J.ri.assign(p.row_indices, p.row_indices + p.num_nonzeros);
  J.val.assign(p.values, p.values + p.num_nonzeros);
  J.cost.assign(p.cost, p.cost + n);
  J.cl.assign(p.col_lower, p.col_lower + n);
  J.cu.assign(p.col_upper, p.col_upper + n);
  J.rl.assign(p.row_lower, p.row_lower + m);
  J.ru.assign(p.row_upper, p.row_upper + m);
  J.view = sankhya_pdhg_problem{m, n, p.num_nonzeros, J.cs.data(), J.ri.data(), J.val.data(),
                                J.cost.data(), J.cl.data(), J.cu.data(), J.rl.data(), J.ru.data(),
                                p.maximize, p.objective_offset};
  const std::string why = validate_model(J.view);
  if (!why.empty()) {
    J.model_error = true;
    J.message = why;
    return;
  }
  if (solo_min_nnz > 0 && J.nnz >= solo_min_nnz) {
    J.solo = true;  // the single-LP engine prepares it itself
    return;
  }
  const double sense = p.maximize ? -1.0 : 1.0;
  std::vector<double> cmin(n);
  double cs2 = 0.0, bs2 = 0.0;
  for (int j = 0; j < n; ++j) {
    cmin[j] = sense * J.cost[j];
    cs2 += cmin[j] * cmin[j];
  }
  for (int i = 0; i < m; ++i) {
    const double b = host_finite_bound(J.rl[i]) ? J.rl[i]
                                                : (host_finite_bound(J.ru[i]) ? J.ru[i] : 0.0);
    bs2 += b * b;
  }
  const Scaling sc = build_scaling(J.view, cmin, 10);
  const PermutedLp q = permute(J.view, sc.values);
  J.group = (cluster_min_nnz > 0 && q.nnz >= cluster_min_nnz) ? kClusterSize : 1;
  const HostPart pa = partition(q.a_ptr, J.group, kWarps, prm.group_size_rows);
  const HostPart pat = partition(q.at_ptr, J.group, kWarps, prm.group_size_cols);
  J.row_perm = q.row_perm;
  J.col_perm = q.col_perm;

  Layout L;
  auto& o = J.off;
  o.a_ptr = L.put((m + 1) * 4);
  o.a_idx = L.put(q.nnz * 4);
  o.a_val = L.put(q.nnz * 8);
  o.at_ptr = L.put((n + 1) * 4);
  o.at_idx = L.put(q.nnz * 4);
  o.at_val = L.put(q.nnz * 8);
  const auto part_off = [&](const HostPart& hp) {
    PartOff po;
    po.blk_seg_begin = L.put(hp.blk_seg_begin.size() * 4);
    po.segs = L.put(hp.segs.size() * 16);
    po.blk_long_begin = L.put(hp.blk_long_begin.size() * 4);
    po.longs = L.put(hp.longs.size() * 16);
    po.blk_item_begin = L.put(hp.blk_item_begin.size() * 4);
    po.items = L.put(hp.items.size() * 16);
    po.seg_sum = L.put(hp.segs.size() * 2 * 8);
    return po;
  };
  o.pa = part_off(pa);
  o.pat = part_off(pat);
  for (size_t* f : {&o.c, &o.cl, &o.cu, &o.dc, &o.c0, &o.cl0, &o.cu0, &o.x0, &o.x1, &o.xsum,
                    &o.xr, &o.xavg, &o.best_x, &o.x_out, &o.red_out, &o.ray_out, &o.xt})
    *f = L.put(n * 8);
  for (size_t* f : {&o.rl, &o.ru, &o.dr, &o.rl0, &o.ru0, &o.y0, &o.y1, &o.ax0, &o.ax1, &o.ysum,
                    &o.yr, &o.yavg, &o.best_y, &o.y_out, &o.farkas_out, &o.yt, &o.axr})
    *f = L.put(m * 8);
  J.image.assign(L.bytes, 0);
  auto& img = J.image;
  write(img, o.a_ptr, q.a_ptr);
  write(img, o.a_idx, q.a_idx);
  write(img, o.a_val, q.a_val);
  write(img, o.at_ptr, q.at_ptr);
  write(img, o.at_idx, q.at_idx);
  write(img, o.at_val, q.at_val);
  const auto part_write = [&](const HostPart& hp, const PartOff& po) {
    write(img, po.blk_seg_begin, hp.blk_seg_begin);
    write(img, po.segs, hp.segs);
    write(img, po.blk_long_begin, hp.blk_long_begin);
    write(img, po.longs, hp.longs);
    write(img, po.blk_item_begin, hp.blk_item_begin);
    write(img, po.items, hp.items);
  };
  part_write(pa, o.pa);
  part_write(pat, o.pat);
  write(img, o.c, gathered(sc.cost, q.col_perm));
  write(img, o.cl, gathered(sc.cl, q.col_perm));
  write(img, o.cu, gathered(sc.cu, q.col_perm));
  write(img, o.rl, gathered(sc.rl, q.row_perm));
  write(img, o.ru, gathered(sc.ru, q.row_perm));
  write(img, o.dr, gathered(sc.dr, q.row_perm));
  write(img, o.dc, gathered(sc.dc, q.col_perm));
  write(img, o.c0, gathered(cmin, q.col_perm));
  write(img, o.cl0, gathered(J.cl, q.col_perm));
  write(img, o.cu0, gathered(J.cu, q.col_perm));
  write(img, o.rl0, gathered(J.rl, q.row_perm));
  write(img, o.ru0, gathered(J.ru, q.row_perm));
  // start: the projection of zero (pdhg.cpp:329-334), also the restart anchor and best point
  std::vector<double> x0(n);
  for (int t = 0; t < n; ++t) {
    const int j = q.col_perm[t];
    double v = 0.0;
    if (host_finite_bound(sc.cl[j]) && v < sc.cl[j]) v = sc.cl[j];
    else if (host_finite_bound(sc.cu[j]) && v > sc.cu[j]) v = sc.cu[j];
    x0[t] = v;
  }
  write(img, o.x0, x0);
  write(img, o.xr, x0);
  write(img, o.best_x, x0);
  // random start of the norm estimate (seed + 1), parked in the average buffer
  std::vector<double> v0(n);
  uniform_draws(static_cast<uint32_t>(prm.random_seed) + 1u, -1.0, 1.0, n, v0.data());
  write(img, o.xavg, gathered(v0, q.col_perm));

  Ctrl& c = J.ctrl0;
  c = Ctrl{};
  c.omega = 1.0;
  c.restart_kkt = INFINITY;
  c.best_worst = INFINITY;
  c.best.primal = c.best.dual = c.best.gap = INFINITY;
  c.state = kSetup;
  c.tolerance = prm.tolerance;
  c.bound_norm = std::sqrt(bs2);
  c.cost_norm = std::sqrt(cs2);
  c.iteration_limit = prm.iteration_limit < 0 ? 1000000ll : prm.iteration_limit;
  c.use_restarts = prm.restart ? 1 : 0;
  c.stop_at_request = prm.stop_at_request ? 1 : 0;
  c.stop_rule = prm.stop_rule;
  c.farkas_cooldown = prm.detect_infeasibility ? 0 : (1 << 30);
  c.halpern = prm.algorithm == SANKHYA_PDHG_ALGORITHM_HALPERN ? 1 : 0;
}

// First-fit allocator over the pool, coalescing on free.
class PoolAllocator {
 public:
  explicit PoolAllocator(size_t bytes) { free_[0] = bytes; }
  bool alloc(size_t bytes, size_t* at) {
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *at = it->first;
        const size_t rest = it->second - bytes, start = it->first + bytes;
        free_.erase(it);
        if (rest) free_[start] = rest;
        used_ += bytes;
        return true;
      }
    }
    return false;
  }
  void release(size_t at, size_t bytes) {
    used_ -= bytes;
    auto it = free_.emplace(at, bytes).first;
    auto next = std::next(it);
    if (next != free_.end() && it->first + it->second == next->first) {
      it->second += next->second;
      free_.erase(next);
    }
    if (it != free_.begin()) {
      auto prev = std::prev(it);
      if (prev->first + prev->second == it->first) {
        prev->second += it->second;
        free_.erase(it);
      }
    }
  }

 private:
  std::map<size_t, size_t> free_;
  size_t used_ = 0;
};

}  // namespace

struct Server {
  sankhya_pdhg_server_config cfg{};
  cudaStream_t stream = nullptr;
  unsigned char* pool = nullptr;
  size_t pool_bytes = 0;
  std::unique_ptr<PoolAllocator> alloc;
  BatchSlot* d_slots = nullptr;
  Ctrl* d_ctrls = nullptr;
  Ctrl* d_compact = nullptr;
  // per class (0: one block per LP, 1: a cluster per LP): active list, count, queue head
  int* d_active[2] = {nullptr, nullptr};
  int* d_count[2] = {nullptr, nullptr};
  int* d_head[2] = {nullptr, nullptr};
  Ctrl* d_compact2 = nullptr;
  Ctrl* h_compact = nullptr;
  Ctrl* h_compact2 = nullptr;
  int* h_active = nullptr;
  int* h_active2 = nullptr;
  int* h_counts = nullptr;
  cudaGraphExec_t graph = nullptr;
  // the split of the GPU between the two classes: clusters for the large LPs, single blocks
  // for the others; chosen per round from the active work, the graph rebuilt when it changes
  int slots_total = 0;     // co-resident blocks of the batch kernels
  int max_clusters = 0;    // co-resident 8-block clusters
  int clusters = 0;        // clusters of the current graph
  int small_grid = 0;      // single blocks of the current graph
  std::vector<int> free_slots;
  std::vector<std::shared_ptr<Job>> slot_job;
  std::vector<int> active;  // slot indices, largest LP first
  std::vector<int> active_big;  // the same for the cluster class
  std::deque<std::shared_ptr<Job>> waiting;
  std::deque<std::shared_ptr<Job>> solo_waiting;  // LPs the single-LP engine solves alone
  std::map<int64_t, std::shared_ptr<Job>> jobs;
  int64_t next_ticket = 1;
  std::mutex mu;
  Clock::time_point t0 = Clock::now();
  long long launches = 0;
  unsigned long long device_clock0 = 0;
  double last_round_seconds = 0.0;  // wall time of the last batched launch
  long long rounds = 0;             // batched launches so far
  // attempts per LP per launch (LPs of at most 16,384 nonzeros per block; larger ones get
  // proportionally fewer): the configured value, or the autotuner's (chunk_attempts = -1)
  long long chunk = 0;
  long long graph_chunk = -1;  // the chunk the current graph was built with
  bool auto_chunk = false;
  int chunk_source = 0;        // 0 configured, 1 tuned here, 2 read from the cache
  std::string chunk_family;    // cache key, once enough LPs have been admitted
  std::vector<long long> family_nnz;
  std::vector<double> family_per_row;
  // the chunk search: LPs finished per second over windows of at least kChunkWindow launches
  // and kChunkWindowSeconds, for every chunk tried
  double round_work = 0.0;     // LPs the last launch finished
  double window_work = 0.0, window_time = 0.0;
  int window_rounds = 0;
  std::map<long long, double> chunk_rate;
  long long best_chunk = 0;
  double best_rate = 0.0;
  int direction = 1;           // 1 doubling, -1 halving
  bool chunk_settled = false;

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

__global__ void read_clock(unsigned long long* out) { *out = global_ns(); }

BatchSlot relocate(const Job& J, unsigned char* base, Ctrl* ctrl) {
  const auto& o = J.off;
  const auto D = [&](size_t off) { return reinterpret_cast<double*>(base + off); };
  const auto I = [&](size_t off) { return reinterpret_cast<int*>(base + off); };
  const auto I4 = [&](size_t off) { return reinterpret_cast<int4*>(base + off); };
  BatchSlot b{};
  Prob<double>& P = b.P;
  P.m = J.m;
  P.n = J.n;
  P.A = Csr<double>{I(o.a_ptr), I(o.a_idx), D(o.a_val), D(o.a_val)};
  P.AT = Csr<double>{I(o.at_ptr), I(o.at_idx), D(o.at_val), D(o.at_val)};
  const auto part = [&](const PartOff& po) {
    return Part{I(po.blk_seg_begin), I4(po.segs), I(po.blk_long_begin), I4(po.longs),
                I(po.blk_item_begin), I4(po.items), D(po.seg_sum)};
  };
  P.pa = part(o.pa);
  P.pat = part(o.pat);
  P.c = D(o.c);
  P.cl = D(o.cl);
  P.cu = D(o.cu);
  P.rl = D(o.rl);
  P.ru = D(o.ru);
  P.dr = D(o.dr);
  P.dc = D(o.dc);
  P.c0 = D(o.c0);
  P.cl0 = D(o.cl0);
  P.cu0 = D(o.cu0);
  P.rl0 = D(o.rl0);
  P.ru0 = D(o.ru0);
  State<double>& S = b.S;
  S.x[0] = D(o.x0);
  S.x[1] = D(o.x1);
  S.y[0] = D(o.y0);
  S.y[1] = D(o.y1);
  S.ax[0] = D(o.ax0);
  S.ax[1] = D(o.ax1);
  S.xsum = D(o.xsum);
  S.ysum = D(o.ysum);
  S.xr = D(o.xr);
  S.yr = D(o.yr);
  S.xavg = D(o.xavg);
  S.yavg = D(o.yavg);
  S.best_x = D(o.best_x);
  S.best_y = D(o.best_y);
  S.xt = D(o.xt);
  S.yt = D(o.yt);
  S.axr = D(o.axr);
  S.partials = nullptr;
  S.ctrl = ctrl;
  b.x_out = D(o.x_out);
  b.red_out = D(o.red_out);
  b.y_out = D(o.y_out);
  b.farkas_out = D(o.farkas_out);
  b.ray_out = D(o.ray_out);
  return b;
}

// Occupancy of the batch kernels: how many blocks, and how many 8-block clusters, fit at once.
void query_capacity(Server& s) {
  int bpsm = 0;
  SIH26_SCUDA(cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)stream_smem_bytes()), SANKHYA_GPU_INIT_FAILED);
  SIH26_SCUDA(cudaFuncSetAttribute(cluster_batch_kernel,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)stream_smem_bytes()), SANKHYA_GPU_INIT_FAILED);
  SIH26_SCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, batch_kernel, kThreads,
                                                            stream_smem_bytes()),
              SANKHYA_GPU_INIT_FAILED);
  cudaDeviceProp props{};
  SIH26_SCUDA(cudaGetDeviceProperties(&props, s.cfg.device), SANKHYA_GPU_INIT_FAILED);
  s.slots_total = props.multiProcessorCount * std::max(1, std::min(bpsm, 2));
  cudaLaunchConfig_t lc{};
  lc.gridDim = dim3(kClusterSize);
  lc.blockDim = dim3(kThreads);
  lc.dynamicSmemBytes = stream_smem_bytes();
  cudaLaunchAttribute attr{};
  attr.id = cudaLaunchAttributeClusterDimension;
  attr.val.clusterDim.x = kClusterSize;
  attr.val.clusterDim.y = 1;
  attr.val.clusterDim.z = 1;
  lc.attrs = &attr;
  lc.numAttrs = 1;
  int max_clusters = 0;
  SIH26_SCUDA(cudaOccupancyMaxActiveClusters(&max_clusters, cluster_batch_kernel, &lc),
              SANKHYA_GPU_INIT_FAILED);
  // keep at least one cluster's worth of blocks for the single-block class
  s.max_clusters = std::max(1, std::min(max_clusters, (s.slots_total - kClusterSize) / kClusterSize));
}

// The round's graph for `clusters` 8-block clusters and the remaining blocks as single blocks:
// the two persistent kernels side by side on two forked streams, then the control blocks of
// both classes compacted for the host.
void build_graph(Server& s, int clusters) {
  clusters = std::max(1, std::min(clusters, s.max_clusters));
  const int small_grid = std::max(1, s.slots_total - clusters * kClusterSize);
  if (s.graph && clusters == s.clusters && small_grid == s.small_grid && s.chunk == s.graph_chunk)
    return;
  if (s.graph) {
    cudaGraphExecDestroy(s.graph);
    s.graph = nullptr;
  }
  cudaStream_t cap, side;
  SIH26_SCUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), SANKHYA_GPU_INIT_FAILED);
  SIH26_SCUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking), SANKHYA_GPU_INIT_FAILED);
  cudaEvent_t fork, join;
  SIH26_SCUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming), SANKHYA_GPU_INIT_FAILED);
  SIH26_SCUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming), SANKHYA_GPU_INIT_FAILED);
  const long long chunk = s.chunk;
  cudaGraph_t g;
  SIH26_SCUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), SANKHYA_GPU_INIT_FAILED);
  cudaMemsetAsync(s.d_head[0], 0, sizeof(int), cap);
  cudaMemsetAsync(s.d_head[1], 0, sizeof(int), cap);
  cudaEventRecord(fork, cap);
  cudaStreamWaitEvent(side, fork, 0);
  cluster_batch_kernel<<<clusters * kClusterSize, kThreads, stream_smem_bytes(), side>>>(
      s.d_slots, s.d_active[1], s.d_count[1], s.d_head[1], chunk);
  gather_ctrl_kernel<<<64, 128, 0, side>>>(s.d_ctrls, s.d_active[1], s.d_count[1], s.d_compact2);
  batch_kernel<<<small_grid, kThreads, stream_smem_bytes(), cap>>>(s.d_slots, s.d_active[0],
                                                                   s.d_count[0], s.d_head[0], chunk);
  gather_ctrl_kernel<<<128, 128, 0, cap>>>(s.d_ctrls, s.d_active[0], s.d_count[0], s.d_compact);
  cudaEventRecord(join, side);
  cudaStreamWaitEvent(cap, join, 0);
  SIH26_SCUDA(cudaStreamEndCapture(cap, &g), SANKHYA_GPU_INIT_FAILED);
  SIH26_SCUDA(cudaGraphInstantiate(&s.graph, g, 0), SANKHYA_GPU_INIT_FAILED);
  cudaGraphDestroy(g);
  cudaEventDestroy(fork);
  cudaEventDestroy(join);
  cudaStreamDestroy(side);
  cudaStreamDestroy(cap);
  s.clusters = clusters;
  s.small_grid = small_grid;
  s.graph_chunk = chunk;
}

// The chunk autotuner (chunk_attempts = -1). Chunking only decides where an LP pauses between
// launches, never what it computes, so the chunk is free to follow measurement. A launch has
// a fixed cost (control blocks, the LPs' start-up, the host round trip) besides its attempts,
// so longer chunks cost less per attempt; but an LP that finishes early in a launch leaves its
// slot idle until the launch ends, so longer chunks also refill the slots of the small LPs
// later. The search measures the served stream's own figure of merit, LPs finished per
// second, over windows of at least kChunkWindow launches and kChunkWindowSeconds, starting at
// kChunkStart and moving by factors of two from the best chunk so far while a step gains more
// than 3 %; when neither neighbour of the best is untried, the best is kept and stored in the
// autotune cache under the family of the first kChunkFamilySample admitted LPs. A chunk cached
// for the family is used as it is.
constexpr long long kChunkMin = 16, kChunkMax = 8192, kChunkStart = 512;
constexpr int kChunkFamilySample = 32, kChunkWindow = 8;
constexpr double kChunkWindowSeconds = 1.0;

void note_family(Server& s, const Job& J) {
  if (!s.auto_chunk || !s.chunk_family.empty()) return;
  s.family_nnz.push_back(J.nnz);
  s.family_per_row.push_back(J.m > 0 ? static_cast<double>(J.nnz) / J.m : 0.0);
  if (static_cast<int>(s.family_nnz.size()) < kChunkFamilySample) return;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s.cfg.device);
  s.chunk_family = chunk_key(sms, s.slots_total, s.family_nnz, s.family_per_row);
  long long cached = 0;
  if (chunk_lookup(autotune_cache_path(), s.chunk_family, &cached)) {
    s.chunk = std::max(kChunkMin, std::min(kChunkMax, cached));
    s.chunk_source = 2;
    s.chunk_settled = true;
  }
}

void tune_chunk(Server& s) {
  if (!s.auto_chunk || s.chunk_settled || s.last_round_seconds <= 0.0) return;
  s.window_work += s.round_work;
  s.window_time += s.last_round_seconds;
  if (++s.window_rounds < kChunkWindow || s.window_time < kChunkWindowSeconds) return;
  const double rate = s.window_work / s.window_time;
  s.window_work = s.window_time = 0.0;
  s.window_rounds = 0;
  s.chunk_rate[s.chunk] = rate;
  if (s.best_chunk == 0 || rate > 1.03 * s.best_rate) {
    s.best_chunk = s.chunk;
    s.best_rate = rate;
  }
  for (int turn = 0; turn < 2; ++turn) {
    const long long next = s.direction > 0 ? s.best_chunk * 2 : s.best_chunk / 2;
    if (next >= kChunkMin && next <= kChunkMax && !s.chunk_rate.count(next)) {
      s.chunk = next;
      return;
    }
    s.direction = -s.direction;
  }
  s.chunk = s.best_chunk;
  s.chunk_settled = true;
  if (!s.chunk_family.empty())
    chunk_store(autotune_cache_path(), s.chunk_family, s.chunk, s.best_rate);  // LPs/s
}

// Clusters for this round: the large class's share of the active nonzeros (its work per
// attempt) of the GPU's blocks, no more than it has LPs, and the configured number when the
// split is fixed (config.clusters > 0 and no adaptation).
int clusters_for_round(const Server& s, long long small_nnz, long long big_nnz, int big_count) {
  if (s.cfg.clusters > 0) return s.cfg.clusters;
  if (big_count == 0) return 1;
  const double share = static_cast<double>(big_nnz) / static_cast<double>(std::max(1ll, small_nnz + big_nnz));
  int want = static_cast<int>(std::lround(share * s.slots_total / kClusterSize));
  want = std::min(want, big_count);
  if (small_nnz > 0) want = std::min(want, s.max_clusters);
  return std::max(1, want);
}

void finish_job(Server& s, Job& J, const Ctrl& c) {
  const int m = J.m, n = J.n;
  const double sense = J.view.maximize ? -1.0 : 1.0;
  unsigned char* base = s.pool + J.pool_offset;
  std::vector<double> hx(n), hred(n), hy(m);
  const auto get = [&](std::vector<double>& v, size_t off) {
    if (!v.empty())
      SIH26_SCUDA(cudaMemcpyAsync(v.data(), base + off, v.size() * 8, cudaMemcpyDeviceToHost,
                                  s.stream), SANKHYA_GPU_COPY_FAILED);
  };
  get(hx, J.off.x_out);
  get(hred, J.off.red_out);
  get(hy, J.off.y_out);
  SIH26_SCUDA(cudaStreamSynchronize(s.stream), SANKHYA_GPU_SYNC_FAILED);
  J.x.assign(n, 0.0);
  J.col_dual.assign(n, 0.0);
  J.row_dual.assign(m, 0.0);
  for (int t = 0; t < n; ++t) {
    J.x[J.col_perm[t]] = hx[t];
    J.col_dual[J.col_perm[t]] = sense * hred[t];
  }
  for (int t = 0; t < m; ++t) J.row_dual[J.row_perm[t]] = sense * (-hy[t]);
  J.last = c;
  const Residuals& f = c.best;
  const bool standard = f.absolute_primal <= 1e-7 && f.absolute_dual <= 1e-7 &&
                        f.gap_as_verified <= 1e-9 && f.complementarity <= 1e-6;
  if (c.state == kInfeasible) {
    J.status = SANKHYA_PDHG_INFEASIBLE;
  } else if (c.state == kUnbounded) {
    // a ray is certified; unboundedness also claims a feasible point for it to start from,
    // which the batched engine does not search for: claimed only when the reported point is
    // feasible to the project's standard (its largest bound violation, measured on the device)
    J.status = c.primal_violation <= 1e-7 ? SANKHYA_PDHG_UNBOUNDED
                                          : SANKHYA_PDHG_INFEASIBLE_OR_UNBOUNDED;
  } else if (c.converged) {
    J.status = standard ? SANKHYA_PDHG_OPTIMAL : SANKHYA_PDHG_FEASIBLE;
  } else {
    J.status = c.state == kTimeLimit ? SANKHYA_PDHG_TIME_LIMIT : SANKHYA_PDHG_ITERATION_LIMIT;
  }
  char msg[256];
  if (J.status == SANKHYA_PDHG_INFEASIBLE) {
    std::snprintf(msg, sizeof msg,
                  "primal infeasible: Farkas certificate from the dual movement after %lld "
                  "iterations (normalised margin %.3e), checked on the original model",
                  c.iteration, c.farkas_margin);
  } else if (J.status == SANKHYA_PDHG_UNBOUNDED) {
    std::snprintf(msg, sizeof msg,
                  "unbounded: primal ray from the last step after %lld iterations, checked on "
                  "the original model",
                  c.iteration);
  } else if (J.status == SANKHYA_PDHG_INFEASIBLE_OR_UNBOUNDED) {
    std::snprintf(msg, sizeof msg,
                  "primal ray from the last step after %lld iterations, checked on the original "
                  "model; the point is not feasible (largest violation %.3e), so unboundedness "
                  "is not claimed",
                  c.iteration, c.primal_violation);
  } else {
    std::snprintf(msg, sizeof msg,
                  "%lld iterations and %lld restarts; relative primal %.3e, dual %.3e, gap %.3e",
                  c.iteration, c.restarts, f.primal, f.dual, f.gap);
  }
  J.message = msg;
  J.finished = true;
  J.finish_time = s.now();
}

}  // namespace

// ---- server operations (called under the server mutex) -----------------------------------

// LPs routed to the single-LP engine, oldest first, each on the whole GPU with its own params,
// between two batched launches (in stream order with the batched work, so the two never share
// the GPU at once): at least one per step and then as many as fit in the time the last batched
// launch took, so either class gets about half of the GPU while both have work; with no
// batched work, up to 16 per step.
static void solve_one_solo(Server& s);

static void run_solo(Server& s) {
  const bool batch_idle = s.active.empty() && s.active_big.empty() && s.waiting.empty();
  const double budget = batch_idle ? 1e30 : s.last_round_seconds;
  const double start = s.now();
  for (int k = 0; k < 16 && !s.solo_waiting.empty(); ++k) {
    if (k > 0 && s.now() - start >= budget) break;
    solve_one_solo(s);
  }
}

static void solve_one_solo(Server& s) {
  std::shared_ptr<Job> J = s.solo_waiting.front();
  s.solo_waiting.pop_front();
  SIH26_SCUDA(cudaStreamSynchronize(s.stream), SANKHYA_GPU_SYNC_FAILED);
  J->admit_time = s.now();
  J->x.assign(J->n, 0.0);
  J->col_dual.assign(J->n, 0.0);
  J->row_dual.assign(J->m, 0.0);
  J->farkas.assign(J->m, 0.0);
  J->ray.assign(J->n, 0.0);
  sankhya_pdhg_result& r = J->solo_result;
  r = sankhya_pdhg_result{};
  r.col_value = J->x.data();
  r.row_dual = J->row_dual.data();
  r.col_dual = J->col_dual.data();
  r.farkas_dual = J->farkas.data();
  r.primal_ray = J->ray.data();
  sankhya_pdhg_params prm = J->prm;
  prm.device = s.cfg.device;
  const int rc = sankhya_pdhg_gpu_solve(&J->view, &prm, &r);
  if (rc != SANKHYA_GPU_SUCCESS) {
    r.status = SANKHYA_PDHG_NUMERICAL_ERROR;
    std::snprintf(r.message, sizeof r.message, "single-LP engine failed: %s",
                  sankhya_pdhg_gpu_last_error());
  }
  if (r.status != SANKHYA_PDHG_INFEASIBLE) J->farkas.clear();
  if (r.status != SANKHYA_PDHG_UNBOUNDED && r.status != SANKHYA_PDHG_INFEASIBLE_OR_UNBOUNDED)
    J->ray.clear();
  J->status = r.status;
  J->message = r.message;
  J->finished = true;
  J->finish_time = s.now();
  s.launches += r.kernel_launches;
}

static void admit(Server& s) {
  bool changed = false;
  while (!s.waiting.empty() && !s.free_slots.empty()) {
    std::shared_ptr<Job> J = s.waiting.front();
    size_t at = 0;
    if (!s.alloc->alloc(J->image.size(), &at)) break;  // no room: wait for retirements
    s.waiting.pop_front();
    const int slot = s.free_slots.back();
    s.free_slots.pop_back();
    J->slot = slot;
    J->pool_offset = at;
    J->pool_bytes = J->image.size();
    J->admit_time = s.now();
    SIH26_SCUDA(cudaMemcpyAsync(s.pool + at, J->image.data(), J->image.size(),
                                cudaMemcpyHostToDevice, s.stream), SANKHYA_GPU_COPY_FAILED);
    Ctrl c = J->ctrl0;
    if (std::isfinite(J->prm.time_limit) && J->prm.time_limit > 0.0) {
      const double since = s.now();
      c.deadline_ns = s.device_clock0 +
                      static_cast<unsigned long long>((since + J->prm.time_limit) * 1e9);
    }
    SIH26_SCUDA(cudaMemcpyAsync(s.d_ctrls + slot, &c, sizeof(Ctrl), cudaMemcpyHostToDevice,
                                s.stream), SANKHYA_GPU_COPY_FAILED);
    const BatchSlot b = relocate(*J, s.pool + at, s.d_ctrls + slot);
    SIH26_SCUDA(cudaMemcpyAsync(s.d_slots + slot, &b, sizeof(BatchSlot), cudaMemcpyHostToDevice,
                                s.stream), SANKHYA_GPU_COPY_FAILED);
    SIH26_SCUDA(cudaStreamSynchronize(s.stream), SANKHYA_GPU_SYNC_FAILED);
    J->image.clear();
    J->image.shrink_to_fit();
    s.slot_job[slot] = J;
    (J->group > 1 ? s.active_big : s.active).push_back(slot);
    note_family(s, *J);
    changed = true;
  }
  if (changed) {
    const auto larger = [&](int a, int b) { return s.slot_job[a]->nnz > s.slot_job[b]->nnz; };
    std::stable_sort(s.active.begin(), s.active.end(), larger);
    std::stable_sort(s.active_big.begin(), s.active_big.end(), larger);
  }
}

// Handles the LPs of one class whose control blocks came back in `compact`; returns those
// still running.
static std::vector<int> settle(Server& s, const std::vector<int>& list, const Ctrl* compact) {
  std::vector<int> still;
  for (size_t q = 0; q < list.size(); ++q) {
    const int slot = list[q];
    const Ctrl& c = compact[q];
    Job& J = *s.slot_job[slot];
    if (c.state == kDeviceError) throw Failure{SANKHYA_GPU_DEVICE_TIMEOUT, "batch kernel error"};
    bool done = c.state == kConverged || c.state == kIterationLimit || c.state == kTimeLimit;
    if (c.state == kInfeasible || c.state == kUnbounded) {
      const bool rows = c.state == kInfeasible;
      const int len = rows ? J.m : J.n;
      std::vector<double> h(len), v(len);
      if (len)
        SIH26_SCUDA(cudaMemcpy(h.data(),
                               s.pool + J.pool_offset + (rows ? J.off.farkas_out : J.off.ray_out),
                               len * 8, cudaMemcpyDeviceToHost), SANKHYA_GPU_COPY_FAILED);
      const std::vector<int>& perm = rows ? J.row_perm : J.col_perm;
      for (int t = 0; t < len; ++t) v[perm[t]] = h[t];
      bool ok = rows ? farkas_holds(J.view, v) : ray_holds(J.view, v);
      if (!ok && !rows && repair_ray(J.view, v)) ok = ray_holds(J.view, v);
      if (ok) {
        (rows ? J.farkas : J.ray) = v;
        done = true;
      } else {
        // not a proof after all: carry on, and give the test a rest
        Ctrl r = c;
        r.state = kRunning;
        r.farkas_cooldown = kCertCooldown;
        SIH26_SCUDA(cudaMemcpyAsync(s.d_ctrls + slot, &r, sizeof(Ctrl), cudaMemcpyHostToDevice,
                                    s.stream), SANKHYA_GPU_COPY_FAILED);
        SIH26_SCUDA(cudaStreamSynchronize(s.stream), SANKHYA_GPU_SYNC_FAILED);
      }
    }
    if (done) {
      s.round_work += 1.0;
      finish_job(s, J, c);
      s.alloc->release(J.pool_offset, J.pool_bytes);
      s.slot_job[slot].reset();
      s.free_slots.push_back(slot);
    } else {
      still.push_back(slot);
    }
  }
  return still;
}

static void run_round(Server& s) {
  const int c0 = static_cast<int>(s.active.size()), c1 = static_cast<int>(s.active_big.size());
  if (c0 + c1 == 0) return;
  long long small_nnz = 0, big_nnz = 0;
  for (int slot : s.active) small_nnz += s.slot_job[slot]->nnz;
  for (int slot : s.active_big) big_nnz += s.slot_job[slot]->nnz;
  int want = clusters_for_round(s, small_nnz, big_nnz, c1);
  // hysteresis: a small change of the ideal split is not worth a new graph
  if (s.graph && std::abs(want - s.clusters) <= std::max(1, s.clusters / 4)) want = s.clusters;
  build_graph(s, want);
  std::memcpy(s.h_active, s.active.data(), c0 * sizeof(int));
  std::memcpy(s.h_active2, s.active_big.data(), c1 * sizeof(int));
  s.h_counts[0] = c0;
  s.h_counts[1] = c1;
  if (c0)
    SIH26_SCUDA(cudaMemcpyAsync(s.d_active[0], s.h_active, c0 * sizeof(int),
                                cudaMemcpyHostToDevice, s.stream), SANKHYA_GPU_COPY_FAILED);
  if (c1)
    SIH26_SCUDA(cudaMemcpyAsync(s.d_active[1], s.h_active2, c1 * sizeof(int),
                                cudaMemcpyHostToDevice, s.stream), SANKHYA_GPU_COPY_FAILED);
  SIH26_SCUDA(cudaMemcpyAsync(s.d_count[0], &s.h_counts[0], sizeof(int), cudaMemcpyHostToDevice,
                              s.stream), SANKHYA_GPU_COPY_FAILED);
  SIH26_SCUDA(cudaMemcpyAsync(s.d_count[1], &s.h_counts[1], sizeof(int), cudaMemcpyHostToDevice,
                              s.stream), SANKHYA_GPU_COPY_FAILED);
  const double started = s.now();
  SIH26_SCUDA(cudaGraphLaunch(s.graph, s.stream), SANKHYA_GPU_KERNEL_LAUNCH_FAILED);
  ++s.launches;
  ++s.rounds;
  if (c0)
    SIH26_SCUDA(cudaMemcpyAsync(s.h_compact, s.d_compact, c0 * sizeof(Ctrl),
                                cudaMemcpyDeviceToHost, s.stream), SANKHYA_GPU_COPY_FAILED);
  if (c1)
    SIH26_SCUDA(cudaMemcpyAsync(s.h_compact2, s.d_compact2, c1 * sizeof(Ctrl),
                                cudaMemcpyDeviceToHost, s.stream), SANKHYA_GPU_COPY_FAILED);
  SIH26_SCUDA(cudaStreamSynchronize(s.stream), SANKHYA_GPU_SYNC_FAILED);
  s.last_round_seconds = s.now() - started;
  s.round_work = 0.0;
  s.active = settle(s, s.active, s.h_compact);
  s.active_big = settle(s, s.active_big, s.h_compact2);
  tune_chunk(s);
}

}  // namespace sih26

// ---- C ABI ----------------------------------------------------------------------------------

using sih26::Failure;
using sih26::Server;

extern "C" {

void sankhya_pdhg_server_default_config(sankhya_pdhg_server_config* c) {
  std::memset(c, 0, sizeof *c);
  c->device = 0;
  c->memory_fraction = 0.8;
  c->pool_bytes = 0;
  c->max_active = 4096;
  c->chunk_attempts = -1;  // the autotuner's (measured against fixed lengths on the served family)
  c->cluster_min_nnz = 16384;
  c->clusters = 0;  // adaptive: the large class's share of the active nonzeros
  c->solo_min_nnz = 0;  // never: routing measured slower on the served family
}

int sankhya_pdhg_server_create(const sankhya_pdhg_server_config* config,
                               sankhya_pdhg_server** out) {
  if (!out) {
    sih26::g_last_error = "out must not be NULL";
    return SANKHYA_GPU_INVALID_ARGUMENT;
  }
  *out = nullptr;
  auto s = std::make_unique<Server>();
  if (config) s->cfg = *config; else sankhya_pdhg_server_default_config(&s->cfg);
  s->auto_chunk = s->cfg.chunk_attempts < 0;
  s->chunk = s->auto_chunk ? sih26::kChunkStart
                           : (s->cfg.chunk_attempts > 0 ? s->cfg.chunk_attempts : (1ll << 40));
  s->chunk_source = s->auto_chunk ? 1 : 0;
  sih26::DeviceGuard guard;
  try {
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0)
      throw Failure{SANKHYA_GPU_NO_COMPATIBLE_DEVICE, "no CUDA device is visible"};
    SIH26_SCUDA(cudaSetDevice(s->cfg.device), SANKHYA_GPU_INIT_FAILED);
    SIH26_SCUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), SANKHYA_GPU_INIT_FAILED);
    size_t free_b = 0, total_b = 0;
    SIH26_SCUDA(cudaMemGetInfo(&free_b, &total_b), SANKHYA_GPU_INIT_FAILED);
    const int cap = s->cfg.max_active > 0 ? s->cfg.max_active : 4096;
    const size_t share =
        static_cast<size_t>(free_b * std::min(0.95, std::max(0.01, s->cfg.memory_fraction)));
    s->pool_bytes = s->cfg.pool_bytes > 0 ? std::min(static_cast<size_t>(s->cfg.pool_bytes), share)
                                          : share;
    s->pool_bytes &= ~size_t(255);
    SIH26_SCUDA(cudaMalloc(&s->pool, s->pool_bytes), SANKHYA_GPU_OUT_OF_MEMORY);
    s->alloc = std::make_unique<sih26::PoolAllocator>(s->pool_bytes);
    SIH26_SCUDA(cudaMalloc(&s->d_slots, cap * sizeof(sih26::BatchSlot)), SANKHYA_GPU_OUT_OF_MEMORY);
    SIH26_SCUDA(cudaMalloc(&s->d_ctrls, cap * sizeof(sih26::Ctrl)), SANKHYA_GPU_OUT_OF_MEMORY);
    SIH26_SCUDA(cudaMalloc(&s->d_compact, cap * sizeof(sih26::Ctrl)), SANKHYA_GPU_OUT_OF_MEMORY);
    for (int k = 0; k < 2; ++k) {
      SIH26_SCUDA(cudaMalloc(&s->d_active[k], cap * sizeof(int)), SANKHYA_GPU_OUT_OF_MEMORY);
      SIH26_SCUDA(cudaMalloc(&s->d_count[k], sizeof(int)), SANKHYA_GPU_OUT_OF_MEMORY);
      SIH26_SCUDA(cudaMalloc(&s->d_head[k], sizeof(int)), SANKHYA_GPU_OUT_OF_MEMORY);
      SIH26_SCUDA(cudaMemsetAsync(s->d_count[k], 0, sizeof(int), s->stream), SANKHYA_GPU_INIT_FAILED);
    }
    SIH26_SCUDA(cudaMalloc(&s->d_compact2, cap * sizeof(sih26::Ctrl)), SANKHYA_GPU_OUT_OF_MEMORY);
    SIH26_SCUDA(cudaMallocHost(&s->h_compact, cap * sizeof(sih26::Ctrl)), SANKHYA_GPU_OUT_OF_MEMORY);
    SIH26_SCUDA(cudaMallocHost(&s->h_compact2, cap * sizeof(sih26::Ctrl)), SANKHYA_GPU_OUT_OF_MEMORY);
    SIH26_SCUDA(cudaMallocHost(&s->h_active, cap * sizeof(int)), SANKHYA_GPU_OUT_OF_MEMORY);
    SIH26_SCUDA(cudaMallocHost(&s->h_active2, cap * sizeof(int)), SANKHYA_GPU_OUT_OF_MEMORY);
    SIH26_SCUDA(cudaMallocHost(&s->h_counts, 2 * sizeof(int)), SANKHYA_GPU_OUT_OF_MEMORY);
    s->slot_job.resize(cap);
    for (int k = cap - 1; k >= 0; --k) s->free_slots.push_back(k);
    sih26::query_capacity(*s);
    sih26::build_graph(*s, s->cfg.clusters > 0 ? s->cfg.clusters : 16);
    unsigned long long* d_clock = nullptr;
    SIH26_SCUDA(cudaMalloc(&d_clock, sizeof *d_clock), SANKHYA_GPU_OUT_OF_MEMORY);
    // freed on every way out of this block, the failing ones included
    std::unique_ptr<unsigned long long, cudaError_t (*)(void*)> clock_owner(d_clock, cudaFree);
    sih26::read_clock<<<1, 1, 0, s->stream>>>(d_clock);
    SIH26_SCUDA(cudaMemcpyAsync(&s->device_clock0, d_clock, sizeof *d_clock,
                                cudaMemcpyDeviceToHost, s->stream), SANKHYA_GPU_COPY_FAILED);
    SIH26_SCUDA(cudaStreamSynchronize(s->stream), SANKHYA_GPU_SYNC_FAILED);
    s->t0 = sih26::Clock::now();
  } catch (const Failure& f) {
    sih26::g_last_error = f.message;
    sankhya_pdhg_server_free(reinterpret_cast<sankhya_pdhg_server*>(s.release()));
    return f.code;
  }
  *out = reinterpret_cast<sankhya_pdhg_server*>(s.release());
  return SANKHYA_GPU_SUCCESS;
}

void sankhya_pdhg_server_free(sankhya_pdhg_server* server) {
  Server* s = reinterpret_cast<Server*>(server);
  if (!s) return;
  sih26::DeviceGuard guard;
  cudaSetDevice(s->cfg.device);
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->graph) cudaGraphExecDestroy(s->graph);
  cudaFree(s->pool);
  cudaFree(s->d_slots);
  cudaFree(s->d_ctrls);
  cudaFree(s->d_compact);
  for (int k = 0; k < 2; ++k) {
    cudaFree(s->d_active[k]);
    cudaFree(s->d_count[k]);
    cudaFree(s->d_head[k]);
  }
  cudaFree(s->d_compact2);
  cudaFreeHost(s->h_compact);
  cudaFreeHost(s->h_compact2);
  cudaFreeHost(s->h_active);
  cudaFreeHost(s->h_active2);
  cudaFreeHost(s->h_counts);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

int sankhya_pdhg_server_submit(sankhya_pdhg_server* server, const sankhya_pdhg_problem* problem,
                               const sankhya_pdhg_params* params, int64_t* ticket) {
  Server* s = reinterpret_cast<Server*>(server);
  if (!s || !problem || !ticket) {
    sih26::g_last_error = "server, problem and ticket must not be NULL";
    return SANKHYA_GPU_INVALID_ARGUMENT;
  }
  sankhya_pdhg_params defaults;
  sankhya_pdhg_gpu_default_params(&defaults);
  auto J = std::make_shared<sih26::Job>();
  try {
    J->submit_time = s->now();
    sih26::prepare(*J, *problem, params ? *params : defaults, s->cfg.cluster_min_nnz,
                   s->cfg.solo_min_nnz);  // host work, outside the lock
  } catch (const Failure& f) {
    sih26::g_last_error = f.message;
    return f.code;
  } catch (const std::bad_alloc&) {
    sih26::g_last_error = "host allocation failed";
    return SANKHYA_GPU_OUT_OF_MEMORY;
  }
  std::lock_guard<std::mutex> lock(s->mu);
  J->ticket = s->next_ticket++;
  *ticket = J->ticket;
  s->jobs[J->ticket] = J;
  if (J->model_error) {
    J->status = SANKHYA_PDHG_MODEL_ERROR;
    J->finished = true;
    J->finish_time = J->submit_time;
  } else if (J->solo) {
    s->solo_waiting.push_back(J);
  } else if (J->image.size() > s->pool_bytes) {
    J->status = SANKHYA_PDHG_NUMERICAL_ERROR;
    J->message = "the LP does not fit the server's device pool";
    J->finished = true;
    J->finish_time = J->submit_time;
  } else {
    s->waiting.push_back(J);
  }
  return SANKHYA_GPU_SUCCESS;
}

int sankhya_pdhg_server_step(sankhya_pdhg_server* server, int32_t* active, int32_t* waiting,
                             int32_t* finished) {
  Server* s = reinterpret_cast<Server*>(server);
  if (!s) {
    sih26::g_last_error = "server must not be NULL";
    return SANKHYA_GPU_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(s->mu);
  sih26::DeviceGuard guard;
  try {
    SIH26_SCUDA(cudaSetDevice(s->cfg.device), SANKHYA_GPU_INIT_FAILED);
    sih26::admit(*s);
    sih26::run_round(*s);
    sih26::admit(*s);
    sih26::run_solo(*s);
  } catch (const Failure& f) {
    sih26::g_last_error = f.message;
    return f.code;
  }
  if (active) *active = static_cast<int32_t>(s->active.size() + s->active_big.size());
  if (waiting) *waiting = static_cast<int32_t>(s->waiting.size() + s->solo_waiting.size());
  if (finished) {
    int32_t k = 0;
    for (auto& kv : s->jobs) k += kv.second->finished ? 1 : 0;
    *finished = k;
  }
  return SANKHYA_GPU_SUCCESS;
}

int sankhya_pdhg_server_get_stats(sankhya_pdhg_server* server, sankhya_pdhg_server_stats* st) {
  Server* s = reinterpret_cast<Server*>(server);
  if (!s || !st) {
    sih26::g_last_error = "server and stats must not be NULL";
    return SANKHYA_GPU_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(s->mu);
  std::memset(st, 0, sizeof *st);
  st->chunk_attempts = s->chunk >= (1ll << 40) ? 0 : s->chunk;
  st->chunk_source = s->chunk_source;
  st->clusters = s->clusters;
  st->rounds = s->rounds;
  st->last_round_ms = s->last_round_seconds * 1e3;
  std::snprintf(st->family, sizeof st->family, "%s", s->chunk_family.c_str());
  return SANKHYA_GPU_SUCCESS;
}

int sankhya_pdhg_server_result(sankhya_pdhg_server* server, int64_t ticket,
                               sankhya_pdhg_result* r) {
  Server* s = reinterpret_cast<Server*>(server);
  if (!s || !r) {
    sih26::g_last_error = "server and result must not be NULL";
    return SANKHYA_GPU_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->jobs.find(ticket);
  if (it == s->jobs.end()) {
    sih26::g_last_error = "unknown ticket";
    return SANKHYA_GPU_INVALID_ARGUMENT;
  }
  sih26::Job& J = *it->second;
  if (!J.finished) return SANKHYA_GPU_NOT_READY;
  if (J.solo) {
    // the single-LP engine's own result, with the caller's arrays and the served times
    sankhya_pdhg_result out = J.solo_result;
    out.col_value = r->col_value;
    out.row_dual = r->row_dual;
    out.col_dual = r->col_dual;
    out.farkas_dual = r->farkas_dual;
    out.primal_ray = r->primal_ray;
    if (out.col_value && !J.x.empty()) std::memcpy(out.col_value, J.x.data(), J.n * 8);
    if (out.col_dual && !J.col_dual.empty()) std::memcpy(out.col_dual, J.col_dual.data(), J.n * 8);
    if (out.row_dual && !J.row_dual.empty()) std::memcpy(out.row_dual, J.row_dual.data(), J.m * 8);
    if (out.farkas_dual && !J.farkas.empty()) std::memcpy(out.farkas_dual, J.farkas.data(), J.m * 8);
    if (out.primal_ray && !J.ray.empty()) std::memcpy(out.primal_ray, J.ray.data(), J.n * 8);
    out.setup_seconds = std::max(0.0, J.admit_time - J.submit_time);
    out.solve_seconds = std::max(0.0, J.finish_time - J.admit_time);
    out.total_seconds = std::max(0.0, J.finish_time - J.submit_time);
    *r = out;
    s->jobs.erase(it);
    return SANKHYA_GPU_SUCCESS;
  }
  r->status = J.status;
  const sih26::Ctrl& c = J.last;
  r->converged = c.converged;
  r->iterations = c.iteration;
  r->attempts = c.attempts;
  r->restarts = c.restarts;
  r->evaluations = c.evaluations;
  r->fp32_iterations = 0;
  r->spectral_norm = c.spectral_norm;
  double obj = J.view.objective_offset;
  for (int j = 0; j < J.n && !J.x.empty(); ++j) obj += J.cost[j] * J.x[j];
  r->objective = obj;
  const sih26::Residuals& f = c.best;
  r->primal_infeasibility = c.primal_violation;
  r->residuals = sankhya_pdhg_residuals{f.primal, f.dual, f.gap, f.primal_objective,
                                        f.dual_objective, f.absolute_primal, f.absolute_dual,
                                        f.gap_as_verified, f.complementarity};
  const double sense = J.view.maximize ? -1.0 : 1.0;
  r->dual_bound = (J.status == SANKHYA_PDHG_OPTIMAL)
                      ? sense * f.dual_objective + J.view.objective_offset
                      : (J.view.maximize ? INFINITY : -INFINITY);
  r->quality = sih26::quality_from_slots(c.quality, r->objective, r->dual_bound);
  r->quality.primal_infeasibility = r->primal_infeasibility;  // one figure for both fields
  if (r->col_value && !J.x.empty()) std::memcpy(r->col_value, J.x.data(), J.n * 8);
  if (r->col_dual && !J.col_dual.empty()) std::memcpy(r->col_dual, J.col_dual.data(), J.n * 8);
  if (r->row_dual && !J.row_dual.empty()) std::memcpy(r->row_dual, J.row_dual.data(), J.m * 8);
  if (r->farkas_dual && !J.farkas.empty()) std::memcpy(r->farkas_dual, J.farkas.data(), J.m * 8);
  if (r->primal_ray && !J.ray.empty()) std::memcpy(r->primal_ray, J.ray.data(), J.n * 8);
  r->setup_seconds = std::max(0.0, J.admit_time - J.submit_time);
  r->solve_seconds = std::max(0.0, J.finish_time - J.admit_time);
  r->total_seconds = std::max(0.0, J.finish_time - J.submit_time);
  r->h2d_bytes = r->d2h_bytes = 0;
  r->iterate_kernel_seconds = 0.0;
  r->iterate_launches = 0;
  r->kernel_launches = s->launches;
  std::snprintf(r->message, sizeof r->message, "%s", J.message.c_str());
  s->jobs.erase(it);
  return SANKHYA_GPU_SUCCESS;
}

int sankhya_pdhg_gpu_batch_solve(const sankhya_pdhg_problem* problems, int32_t count,
                                 const sankhya_pdhg_params* params, sankhya_pdhg_result* results) {
  if (count < 0 || (count > 0 && (!problems || !results))) {
    sih26::g_last_error = "problems and results must hold count entries";
    return SANKHYA_GPU_INVALID_ARGUMENT;
  }
  sankhya_pdhg_server_config cfg;
  sankhya_pdhg_server_default_config(&cfg);
  if (params) cfg.device = params->device;
  cfg.chunk_attempts = 0;  // run every LP to its end in one launch
  // a pool just large enough for every image at once (an upper bound of the layout of
  // prepare(): 24 bytes per nonzero for both orientations, 17 FP64 vectors per row and per
  // column, the work partitions and alignment), instead of a share of all free memory
  {
    size_t bound = size_t(64) << 20;
    for (int k = 0; k < count; ++k) {
      const sankhya_pdhg_problem& q = problems[k];
      if (q.num_rows < 0 || q.num_cols < 0 || q.num_nonzeros < 0) continue;
      bound += 26 * static_cast<size_t>(q.num_nonzeros) +
               200 * (static_cast<size_t>(q.num_rows) + static_cast<size_t>(q.num_cols)) +
               (size_t(64) << 10);
    }
    cfg.pool_bytes = static_cast<int64_t>(bound);
  }
  sankhya_pdhg_server* server = nullptr;
  int rc = sankhya_pdhg_server_create(&cfg, &server);
  if (rc != SANKHYA_GPU_SUCCESS) return rc;
  // host preparation (validation, scaling, layout) of the LPs on several threads; submit is
  // thread-safe and the results do not depend on the order of admission
  std::vector<int64_t> tickets(count);
  std::vector<int> codes(count, SANKHYA_GPU_SUCCESS);
  std::vector<std::string> errors(count);
  {
    const int workers = std::max(1, std::min<int>(count, std::min(16u, std::max(1u, std::thread::hardware_concurrency()))));
    std::atomic<int> next{0};
    std::vector<std::thread> pool;
    for (int w = 0; w < workers; ++w) {
      pool.emplace_back([&] {
        for (int k = next++; k < count; k = next++) {
          codes[k] = sankhya_pdhg_server_submit(server, &problems[k], params, &tickets[k]);
          if (codes[k] != SANKHYA_GPU_SUCCESS) errors[k] = sih26::g_last_error;
        }
      });
    }
    for (auto& t : pool) t.join();
  }
  for (int k = 0; k < count; ++k) {
    if (codes[k] != SANKHYA_GPU_SUCCESS) {
      rc = codes[k];
      sih26::g_last_error = errors[k];
      break;
    }
  }
  int32_t active = 0, waiting = 0, finished = 0;
  while (rc == SANKHYA_GPU_SUCCESS) {
    rc = sankhya_pdhg_server_step(server, &active, &waiting, &finished);
    if (active == 0 && waiting == 0) break;
  }
  for (int k = 0; k < count && rc == SANKHYA_GPU_SUCCESS; ++k)
    rc = sankhya_pdhg_server_result(server, tickets[k], &results[k]);
  sankhya_pdhg_server_free(server);
  return rc;
}

}  // extern "C"
