/* SANKHYA restarted-PDHG LP engine on one NVIDIA B200 (sm_100a) -- C ABI.
 *
 * This is the drop-in for the reference solver's CPU PDHG call
 *     Solution sankhya::pdhg::solve_pdhg(const Model&, const Options&, Logger&)
 *     (include/sankhya/pdhg.hpp:15, src/pdhg/pdhg.cpp:267-726)
 * at its one call site, run_lp_engine in src/core/solve.cpp:385-395. The adapter a maintainer
 * adds on the reference side turns the Model and Options into the structs below and the
 * result back into a Solution; it is shown in INTEGRATION.md.
 *
 * Conventions follow the reference's C API (include/sankhya/sankhya.h:16-28):
 *   ERRORS are returned, never thrown; sankhya_pdhg_gpu_last_error() gives the reason for the
 *     most recent failing call on the calling thread.
 *   OWNERSHIP: the caller owns every input array and every output buffer; the library owns
 *     device memory and handles, released by the matching *_free.
 *   THREADING: a handle is not internally synchronised; distinct handles on distinct threads
 *     are fine. The error string is thread-local.
 *   NO CPU FALLBACK: when the GPU path cannot run, the call fails with a status; nothing is
 *     silently computed on the host.
 *
 * Storage matches the reference's SparseMatrix (include/sankhya/sparse.hpp:109-112): CSC,
 * int32 column starts [n+1] and row indices [nnz] ascending within each column, FP64 values.
 * An absent bound is +-inf or any |v| >= 1e30 (include/sankhya/types.hpp:32-39).
 */
#ifndef SANKHYA_PDHG_GPU_H
#define SANKHYA_PDHG_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Status of a call. The values mirror sankhya::gpu::GpuStatus
 *      (include/sankhya/gpu_runtime.hpp:19-30); 10 and 11 are additions. ------------------ */
typedef enum sankhya_pdhg_gpu_status {
  SANKHYA_GPU_SUCCESS = 0,
  SANKHYA_GPU_CUDA_UNAVAILABLE = 1,
  SANKHYA_GPU_NO_COMPATIBLE_DEVICE = 2,
  SANKHYA_GPU_INIT_FAILED = 3,
  SANKHYA_GPU_OUT_OF_MEMORY = 4,
  SANKHYA_GPU_KERNEL_LAUNCH_FAILED = 5,
  SANKHYA_GPU_COPY_FAILED = 6,
  SANKHYA_GPU_SYNC_FAILED = 7,
  SANKHYA_GPU_INVALID_DEVICE_STATE = 8,
  SANKHYA_GPU_NON_FINITE_OUTPUT = 9,
  SANKHYA_GPU_INVALID_ARGUMENT = 10, /* malformed problem or parameters; see last_error */
  SANKHYA_GPU_DEVICE_TIMEOUT = 11,   /* a bounded device-side wait gave up; context intact */
  SANKHYA_GPU_NOT_READY = 12         /* server: the LP has not finished yet */
} sankhya_pdhg_gpu_status;

/* ---- Solve status of a result: the values of sankhya_solve_status
 *      (include/sankhya/sankhya.h:53-66). ---------------------------------------------- */
enum {
  SANKHYA_PDHG_NOT_SOLVED = 0,
  SANKHYA_PDHG_OPTIMAL = 1,
  SANKHYA_PDHG_FEASIBLE = 2,
  SANKHYA_PDHG_INFEASIBLE = 3,
  SANKHYA_PDHG_UNBOUNDED = 4,
  SANKHYA_PDHG_ITERATION_LIMIT = 5,
  SANKHYA_PDHG_TIME_LIMIT = 6,
  SANKHYA_PDHG_NUMERICAL_ERROR = 8,
  SANKHYA_PDHG_MODEL_ERROR = 9,
  /* a certified primal ray (the LP has no bounded optimum) without a point shown to be
     feasible, so unboundedness is not claimed (SANKHYA_INFEASIBLE_OR_UNBOUNDED) */
  SANKHYA_PDHG_INFEASIBLE_OR_UNBOUNDED = 10
};

/* Arithmetic of the iteration. */
enum {
  SANKHYA_PDHG_FP64 = 0,  /* FP64 matrix, iterates and reductions throughout */
  SANKHYA_PDHG_MIXED = 1  /* FP32 matrix and FP32 iterate deltas about an FP64 restart
                             anchor, FP64 reductions and FP64 KKT, restart and step-size
                             logic; an FP64 polish phase takes over from the FP32 state when
                             the FP32 level stops improving before the request */
};

/* Stopping rule. */
enum {
  /* src/pdhg/pdhg.cpp:585-586: meets_request(tol) AND (stop_at_request OR the project's
   * absolute standard: primal 1e-7, dual 1e-7, verified gap 1e-9, complementarity 1e-6). */
  SANKHYA_PDHG_STOP_REFERENCE = 0,
  /* Relative KKT only: max(relative primal, relative dual, relative gap) <= tolerance, the
   * PDLP-literature criterion (time-to-relative-KKT). Status is still assigned by the
   * reference's rules (optimal only when the absolute standard holds). */
  SANKHYA_PDHG_STOP_RELATIVE_KKT = 1
};

/* Iteration operator (single-LP path). */
enum {
  /* src/pdhg/pdhg.cpp:383-644: adaptive step size with acceptance test, running average,
   * restarts on the KKT error (sufficient 0.2, artificial 0.36 of the iterations), primal
   * weight smoothing 0.5. */
  SANKHYA_PDHG_ALGORITHM_REFERENCE = 0,
  /* Reflected restarted Halpern PDHG (Lu & Yang, "Restarted Halpern PDHG for linear
   * programming", 2024): z_{k+1} = (k+1)/(k+2) (2 T(z_k) - z_k) + 1/(k+2) z_0 with T one PDHG
   * step at the constant step size 0.998/||A||_2 and z_0 the last restart point. The
   * candidates, restart rules, primal weight, stopping test and status rules stay the
   * reference's; the PDHG output T(z_k) takes the place of the running average. */
  SANKHYA_PDHG_ALGORITHM_HALPERN = 1
};

/* One LP as the reference's Model holds it (include/sankhya/model.hpp:131-225). */
typedef struct sankhya_pdhg_problem {
  int32_t num_rows;
  int32_t num_cols;
  int32_t num_nonzeros;
  const int32_t* col_starts;  /* [n+1] */
  const int32_t* row_indices; /* [nnz] */
  const double* values;       /* [nnz] */
  const double* cost;         /* [n], in the model's own sense */
  const double* col_lower;    /* [n] */
  const double* col_upper;    /* [n] */
  const double* row_lower;    /* [m] */
  const double* row_upper;    /* [m] */
  int32_t maximize;           /* model.sense == kMaximize */
  double objective_offset;
} sankhya_pdhg_problem;

/* Options. Fill with sankhya_pdhg_gpu_default_params(); the first six mirror the reference's
 * option registry rows of the same name (src/util/options.cpp:83-418). */
typedef struct sankhya_pdhg_params {
  double tolerance;         /* pdhg_tolerance, default 1e-4 */
  int64_t iteration_limit;  /* iteration_limit, -1 = 1,000,000 (src/pdhg/pdhg.cpp:311-313) */
  double time_limit;        /* time_limit in seconds, default +inf */
  int32_t restart;          /* pdhg_restart, default 1 */
  int32_t stop_at_request;  /* pdhg_stop_at_request, default 0 */
  int64_t random_seed;      /* random_seed, default 0 (the norm estimate uses seed + 1) */
  /* GPU knobs (new rows) */
  int32_t precision;        /* SANKHYA_PDHG_FP64 (default) or SANKHYA_PDHG_MIXED */
  int32_t stop_rule;        /* SANKHYA_PDHG_STOP_REFERENCE (default) or _RELATIVE_KKT */
  int32_t device;           /* CUDA device ordinal, default 0 */
  int32_t verbose;          /* 1 prints the iteration table at each evaluation */
  int32_t detect_infeasibility; /* 1 (default): certify primal infeasibility / dual
                                   unboundedness from iterate differences */
  double mixed_switch_tolerance; /* MIXED: relative KKT at which the FP32 phase hands over to
                                    the FP64 polish (with its whole restart state); 0 (default)
                                    = the request (no finer than 1e-10), or earlier if the FP32
                                    level stops improving */
  int32_t group_size_rows;  /* lanes per row for A x (0 = autotune) */
  int32_t group_size_cols;  /* lanes per row for A'y (0 = autotune) */
  int32_t grid_blocks;      /* blocks of the cooperative launches (0 = sized to the problem) */
  int32_t profile_kernels;  /* 1: time every iteration-kernel launch with CUDA events */
  int32_t mixed_stall_checks; /* MIXED: host checks (about 2,600 iterations each) without a
                                 better KKT error before the FP32 phase hands over; 0 = auto
                                 (no 1% gain over the last 30% of the iterations), -1 = never */
  int32_t algorithm;        /* SANKHYA_PDHG_ALGORITHM_REFERENCE (default) or _HALPERN */
  int32_t autotune;         /* 1: pick the SpMV schedule of A and A' (rows per stream item,
                               nonzeros per lane) by timing candidates on this LP, keyed on its
                               row-length statistics and cached on disk
                               (SANKHYA_PDHG_AUTOTUNE_CACHE, else ~/.cache/sih26_b200/
                               autotune.tsv); 0 (default): the fixed rule */
  int32_t prep;             /* where the LP is scaled and laid out: 0 (default) on the device
                               from 100,000 nonzeros and on the host below (per-call launch
                               costs dominate there), 1 always on the host, 2 always on the
                               device. All give identical bits. */
  int32_t qp_assume_convex; /* QP only: 1 skips the convexity test (for QPs beyond its
                                2,000-column limit whose convexity the caller knows) */
  int32_t reserved[1];
} sankhya_pdhg_params;

/* Unscaled residual block of the reported point (src/pdhg/pdhg.cpp:81-110). */
typedef struct sankhya_pdhg_residuals {
  double relative_primal;
  double relative_dual;
  double relative_gap;
  double primal_objective; /* minimise space, offset excluded */
  double dual_objective;
  double absolute_primal;
  double absolute_dual;
  double gap_as_verified;
  double complementarity;
} sankhya_pdhg_residuals;

/* Result. The caller allocates the arrays (any may be NULL); the library fills the rest.
 * Sign conventions follow src/pdhg/pdhg.cpp:647-661: row_dual = sense * (-y),
 * col_dual = sense * (c_min + A'y), with y the PDHG multiplier. */
/* Quality of the reported point, as Solution::recompute_quality (src/core/model.cpp:228-424)
 * measures it, computed on the device from the reported x, row_dual and col_dual in original
 * units. The same definitions term by term; only the rounding of the row and column sums
 * differs from the host code's. LP solves fill every field; the QP solve fills
 * primal_infeasibility only and sets the other fields to NaN. */
typedef struct sankhya_pdhg_quality {
  double primal_infeasibility;        /* max violation over row and column bounds */
  double primal_infeasibility_scaled; /* each violation over its quantity's term scale */
  double dual_infeasibility;          /* max reduced-cost / row-price sign violation and
                                         max |c - A'row_dual - col_dual| */
  double dual_infeasibility_scaled;   /* the same (and complementarity) over their scales */
  double complementarity_violation;   /* max |multiplier| * distance to the nearest bound */
  double absolute_gap;                /* |objective - dual_bound| */
  double relative_gap;                /* absolute_gap / max(1, |objective|) */
} sankhya_pdhg_quality;

typedef struct sankhya_pdhg_result {
  double* col_value;   /* [n]; for UNBOUNDED a feasible point the ray starts from */
  double* row_dual;    /* [m] */
  double* col_dual;    /* [n] */
  double* farkas_dual; /* [m] filled when status is INFEASIBLE (row_dual sign) */
  double* primal_ray;  /* [n] filled when status is UNBOUNDED or INFEASIBLE_OR_UNBOUNDED */
  int32_t status;      /* SANKHYA_PDHG_* solve status */
  int32_t converged;
  int64_t iterations;  /* accepted iterations, all phases */
  int64_t attempts;    /* accepted + rejected steps */
  int64_t restarts;
  int64_t evaluations;
  int64_t fp32_iterations; /* MIXED: accepted iterations in the FP32 phase */
  double objective;    /* original sense, offset included */
  double dual_bound;   /* finite only when the point meets the project standard */
  double spectral_norm;
  double setup_seconds;  /* validation, scaling, upload, norm estimate */
  double solve_seconds;  /* the iteration loop, device-timed */
  double total_seconds;  /* the whole call, host wall clock */
  int64_t h2d_bytes;     /* host -> device bytes copied by the call */
  int64_t d2h_bytes;     /* device -> host bytes copied by the call */
  double iterate_kernel_seconds; /* profile_kernels: summed event-timed iteration launches */
  int64_t iterate_launches;      /* profile_kernels: how many were timed */
  int64_t kernel_launches;       /* every kernel this call launched */
  sankhya_pdhg_residuals residuals;
  int32_t autotuned;    /* 0 fixed rule, 1 schedule measured by this call, 2 read from cache */
  int32_t schedule[4];  /* stream-row limit and nonzeros per lane of A, then of A' */
  double primal_infeasibility; /* largest bound violation of col_value and of A col_value,
                                  in original units (Solution::recompute_quality,
                                  src/core/model.cpp:228-283), computed on the device */
  sankhya_pdhg_quality quality; /* the whole recompute_quality block of the reported point */
  char message[512];
} sankhya_pdhg_result;

/* Defaults equal to the reference's option defaults. */
void sankhya_pdhg_gpu_default_params(sankhya_pdhg_params* params);

/* Solve one LP on the GPU. Replaces pdhg::solve_pdhg (src/pdhg/pdhg.cpp:267) for the
 * adapter at src/core/solve.cpp:392. A model the reference would reject (Model::validate,
 * src/core/model.cpp:125-210) returns SUCCESS with status MODEL_ERROR and the reason in
 * result->message, as solve_pdhg does (src/pdhg/pdhg.cpp:273-278). */
int sankhya_pdhg_gpu_solve(const sankhya_pdhg_problem* problem,
                           const sankhya_pdhg_params* params, sankhya_pdhg_result* result);

/* Unscaled KKT residuals of a point, on the GPU, without allocating any memory.
 *
 * This entry point has no counterpart in the reference. It exists for callers that cannot
 * allocate device memory while they run: an application whose device memory belongs to its
 * own pool or arena and forbids raw cudaMalloc/cudaFree, a service that fixes its device
 * budget at start-up, or a latency-critical loop that cannot afford the device-wide
 * synchronisation cudaMalloc/cudaFree imply. It computes the residual block of
 * src/pdhg/pdhg.cpp:143-263 (the same definitions sankhya_pdhg_gpu_solve reports in
 * result->residuals) for the point (x, row_dual) of the LP `problem`.
 *
 * Every pointer inside `problem`, and x[n], row_dual[m] (reference sign: sense * -y) and
 * residuals_out[9] (written in sankhya_pdhg_residuals field order), are DEVICE pointers on
 * the current device; the struct itself is read on the host. Work is queued on `stream`
 * (a cudaStream_t; NULL = the legacy default stream) and residuals_out is valid once that
 * stream reaches it. An out-of-range row index makes every output NaN. A x is accumulated
 * with FP64 atomic adds, so the last bits of the outputs can differ from call to call; every
 * other entry point of this library is bit-for-bit repeatable.
 *
 * Scratch is a fixed 4 MiB device array inside the library (held by every GPU that loads
 * it until the process exits), so problems with more than SANKHYA_PDHG_NOALLOC_MAX_ROWS rows
 * are rejected with SANKHYA_GPU_INVALID_ARGUMENT. Every call looks up the array's device
 * address on the current device (cudaGetSymbolAddress, which allocates nothing); the first
 * call on a device is also the one that loads the library's device code there, so make it
 * before any stream capture. All calls share the array and each leaves its contents behind
 * (each clears what it needs zeroed before use): calls whose work overlaps on the GPU race and
 * must be ordered on one stream. Nothing is allocated, host or device. */
#define SANKHYA_PDHG_NOALLOC_MAX_ROWS 516064
int sankhya_pdhg_gpu_residuals_noalloc(const sankhya_pdhg_problem* problem, const double* x,
                                       const double* row_dual, double* residuals_out,
                                       void* stream);

/* ---- Many LPs at once: the served / batched engine ------------------------------------
 *
 * A server keeps LPs resident on one GPU and runs every admitted LP in one persistent kernel
 * launch per step: each thread block takes LPs from a device work queue (largest first) and
 * runs the restarted PDHG of src/pdhg/pdhg.cpp on one LP with its own step size, primal
 * weight, restarts, termination and norm estimate, for at most chunk_attempts attempts per
 * step. LPs submitted while others run are admitted between steps when their device image
 * fits the memory pool (a fraction of free HBM taken at creation) and join the next launch;
 * finished LPs are retired with their answers. Primal infeasibility is certified from the
 * dual movement between restarts and every certificate is re-checked on the host against
 * the original model (the test of src/core/certificate.cpp:29-119) before it is reported.
 * These entry points are the batch / server successors the reference's GPU slot never had. */
typedef struct sankhya_pdhg_server sankhya_pdhg_server;

typedef struct sankhya_pdhg_server_config {
  int32_t device;          /* CUDA device ordinal */
  double memory_fraction;  /* share of free device memory for the pool (default 0.8) */
  int64_t pool_bytes;      /* explicit pool size; 0 = use memory_fraction */
  int32_t max_active;      /* LP slots (default 4096) */
  int64_t chunk_attempts;  /* attempts per LP per step for LPs with at most 16,384 nonzeros
                              per block; larger LPs get proportionally fewer (at least 8), so
                              a step lasts about as long for every LP; 0 = run each LP to its
                              end; -1 (default) = autotuned: a search over powers of two
                              (16-8,192) for the most LPs finished per second (over windows of
                              at least 8 launches and 1 s), starting from 512 or, once 32 LPs
                              have been admitted, from the value the autotune cache (see
                              sankhya_pdhg_params.autotune) holds for their family (keyed on
                              the SM count, the launch slots and the LPs' median nonzeros and
                              nonzeros per row); the value it settles on is stored there.
                              Chunking only pauses an LP between launches: its answer is the
                              same for every chunk length */
  int64_t cluster_min_nnz; /* LPs with at least this many nonzeros run on an 8-block thread
                              block cluster instead of one block (default 16384; 0 = never) */
  int32_t clusters;        /* clusters for those LPs; 0 (default): chosen every round from
                              the large LPs' share of the active nonzeros (the rest of the GPU
                              runs the small LPs on single blocks) */
  int32_t solo_min_nnz;    /* LPs with at least this many nonzeros are solved one at a time on
                              the whole GPU by the single-LP engine (sankhya_pdhg_gpu_solve with
                              the LP's own params) between the batched launches, for as long as
                              the last batched launch took; 0 (default) = never: on the served
                              family the batched engine's clusters served the large LPs faster */
  int32_t reserved[6];
} sankhya_pdhg_server_config;

/* A server's current launch settings. */
typedef struct sankhya_pdhg_server_stats {
  int64_t chunk_attempts; /* attempts per LP per launch in use now (0 = each LP to its end) */
  int32_t chunk_source;   /* 0 configured, 1 tuned by this server (searching or settled),
                             2 read from the cache */
  int32_t clusters;       /* 8-block clusters of the current launch graph */
  int64_t rounds;         /* batched launches so far */
  double last_round_ms;   /* wall time of the last batched launch */
  char family[192];       /* chunk_attempts = -1: the autotune cache key of the admitted LPs'
                             family, once 32 have been admitted ("" before) */
  int32_t reserved[4];
} sankhya_pdhg_server_stats;

void sankhya_pdhg_server_default_config(sankhya_pdhg_server_config* config);
int sankhya_pdhg_server_create(const sankhya_pdhg_server_config* config,
                               sankhya_pdhg_server** server);
/* Prepares the LP on the host (validation, scaling, layout) and queues it; thread-safe. */
int sankhya_pdhg_server_submit(sankhya_pdhg_server* server, const sankhya_pdhg_problem* problem,
                               const sankhya_pdhg_params* params, int64_t* ticket);
/* Admits what fits, runs one launch over every active LP, retires the finished ones. */
int sankhya_pdhg_server_step(sankhya_pdhg_server* server, int32_t* active, int32_t* waiting,
                             int32_t* finished);
/* SANKHYA_GPU_NOT_READY until the LP has finished; then fills `result` (the caller's arrays,
 * as for sankhya_pdhg_gpu_solve, plus farkas_dual for INFEASIBLE) and forgets the ticket.
 * setup_seconds / solve_seconds / total_seconds are queueing, device and submit-to-finish
 * times. */
int sankhya_pdhg_server_result(sankhya_pdhg_server* server, int64_t ticket,
                               sankhya_pdhg_result* result);
void sankhya_pdhg_server_free(sankhya_pdhg_server* server);
/* Fills *stats with the server's current launch settings. */
int sankhya_pdhg_server_get_stats(sankhya_pdhg_server* server, sankhya_pdhg_server_stats* stats);

/* Solves `count` independent LPs concurrently on one GPU (a server, every LP submitted, run
 * to the end, results collected). results[k] is filled like sankhya_pdhg_gpu_solve's. */
int sankhya_pdhg_gpu_batch_solve(const sankhya_pdhg_problem* problems, int32_t count,
                                 const sankhya_pdhg_params* params, sankhya_pdhg_result* results);

/* ---- Convex QP ------------------------------------------------------------------------------
 *
 * min 0.5 x'Qx + c'x (in the model's sense) over the same constraints, by the reference's
 * Condat-Vu primal-dual method (src/qp/qp_condat_vu.cpp:150-323): the LP engine's primal step
 * plus the gradient Qx, fixed steps from power-iteration estimates of ||A|| and ||Q||,
 * termination on max-norm primal and projected-gradient residuals every 50 iterations. Q is
 * given as its lower triangle in CSC (the reference's Model::hessian, model.hpp:156); the
 * 0.5 lives in the objective, so an off-diagonal entry stands for two entries of Q. */
typedef struct sankhya_qp_hessian {
  int32_t num_nonzeros;
  const int32_t* col_starts;  /* [n+1], n = problem->num_cols */
  const int32_t* row_indices; /* [nnz], row >= column, ascending within a column */
  const double* values;       /* [nnz] */
} sankhya_qp_hessian;

/* Replaces qp::solve_convex_qp (src/qp/qp_condat_vu.cpp:150). params->tolerance is the
 * reference's qp_tolerance (default 1e-8 when params->tolerance <= 0); iteration_limit,
 * time_limit and device as for sankhya_pdhg_gpu_solve. Like the reference, a Q that is not
 * convex in minimisation sense -- or whose convexity the dense test (n <= 2,000,
 * src/qp/convexity.cpp:17-136) cannot decide -- returns SUCCESS with status MODEL_ERROR,
 * unless params->qp_assume_convex is 1. Fills col_value, row_dual (= -sense y), col_dual
 * (= c + Qx + sense A'y, as the reference), objective (with the quadratic term), status,
 * iterations, the residual block's absolute_primal / absolute_dual (the two termination
 * measures), primal_infeasibility and message. */
int sankhya_qp_gpu_solve(const sankhya_pdhg_problem* problem, const sankhya_qp_hessian* hessian,
                         const sankhya_pdhg_params* params, sankhya_pdhg_result* result);

/* ---- Request wire format -----------------------------------------------------------------
 *
 * A binary form of one LP for served mode, where parsing text MPS per request would cost more
 * than solving (the reference reads MPS/LP text, src/io/mps_reader.cpp; this format has no
 * counterpart there). Little-endian, every array 8-byte aligned so a received buffer is used
 * in place:
 *   0  char[8]  "SKPDHG01"
 *   8  int32    num_rows, num_cols, num_nonzeros, flags (bit 0: maximize)
 *   24 double   objective_offset
 *   32 arrays   col_starts[n+1] int32, row_indices[nnz] int32, values[nnz], cost[n],
 *               col_lower[n], col_upper[n], row_lower[m], row_upper[m] (doubles), each
 *               starting on an 8-byte boundary (int32 arrays padded with zeros). */
#define SANKHYA_PDHG_WIRE_MAGIC "SKPDHG01"

/* Bytes the wire form of `problem` takes. */
size_t sankhya_pdhg_wire_size(const sankhya_pdhg_problem* problem);
/* Writes the wire form of `problem` into buffer[0, bytes); INVALID_ARGUMENT if it does not
 * fit or the problem is malformed. */
int sankhya_pdhg_wire_write(const sankhya_pdhg_problem* problem, void* buffer, size_t bytes);
/* Points `problem` into a wire buffer without copying (the buffer must stay alive and be
 * 8-byte aligned); checks the magic, the sizes against `bytes` and the CSC structure, and
 * returns INVALID_ARGUMENT with the reason in last_error otherwise. */
int sankhya_pdhg_wire_view(const void* buffer, size_t bytes, sankhya_pdhg_problem* problem);

/* Reason for the most recent failing call on this thread (never NULL). */
const char* sankhya_pdhg_gpu_last_error(void);

/* Device queries, the successors of is_cuda_available / get_gpu_device_count
 * (include/sankhya/gpu_runtime.hpp:71-77). */
int sankhya_pdhg_gpu_device_count(void);
int sankhya_pdhg_gpu_device_name(int device, char* name, int capacity);

#ifdef __cplusplus
}
#endif

#endif /* SANKHYA_PDHG_GPU_H */
