"""Benchmark: time to relative KKT 1e-6 of the GPU restarted PDHG, FP32-mixed vs FP64.

Workload (one LP): 200,000 rows x 500,000 columns, 10 nonzeros per column (5M), rows drawn
by Pareto(1.5) weights so some rows hold thousands of entries, values N(0,1) x 10^U(-2,2)
per row, equality rows, 0 <= x <= u, planted optimum (sih26_b200.lpgen.powerlaw_planted,
seed 1). A step is one solve to relative KKT 1e-6 (max of relative primal, dual and gap,
FP64, unscaled) through the library's C ABI.

  value   device seconds of the iteration loop (CUDA events on the solve's stream; the LP
          was uploaded, scaled and its norm estimated before the timed region), FP32-mixed,
          with the iteration operator of --algorithm (default: the Halpern operator; the
          reference's operator is timed once in each precision beside it)
  e2e     the same solve measured around the public call with host arrays: validation,
          host scaling, H2D of the problem, the loop, D2H of x / y / reduced costs
  fp64    the same metric on the plain FP64 path
  roofline  the iteration kernel (the dominant kernel): algorithmic bytes per attempt x
          attempts / event-timed launch durations, against the measured HBM copy bandwidth
  cpu_baseline  the reference's own solve_pdhg built from its sources (oracle/_ref), all host
          threads, on a bounded sample: setup + 20 iterations, extrapolated to the iteration
          count of this workload

  batched  512 uneven LPs (m log-uniform on [50, 5,000], n = m U(1.5, 3), 5-15 nonzeros per
          column, 10 % primal-infeasible; lpgen.uneven_batch, seed 3) solved to relative KKT
          1e-6 by the batched engine in one call (sankhya_pdhg_gpu_batch_solve, host arrays in
          and out): LPs/s, p50 / p99 / p99.9 submit-to-answer latency, certificates found, and
          the same LPs solved one at a time by the plain FP64 single-LP path (a sample of every
          8th LP) for the LPs/s ratio. Under torchrun the 512 LPs are sharded by nonzeros
          (sih26_b200.shard) and the time is the maximum over ranks.
  served  Poisson request streams (default 50 and 200 LPs/s for 4 s; LPs drawn from a seeded pool of
          the served family, m log-uniform on [100, 50,000]) into a resident server that admits
          requests between launches of its persistent kernels (continuous batching): LPs/s and
          p50 / p99 / p99.9 arrival-to-answer latency, next to one-at-a-time FP64 solves of
          the same pool. Rank 0 only.

  qp      the convex-QP engine on a planted 800 x 2,000 QP next to the reference's own QP
          engine on the host, and on a 40,000 x 100,000 QP alone (rank 0 only).

`--impl reference` times that CPU reference alone on the same workload and prints its line.
With torchrun (N > 1) every rank solves its own replica of the LP (a single LP does not
shard); the time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

TOLERANCE = 1e-6
SEED = 1
REF_SAMPLE_ITERATIONS = 20
# Iterations the FP64 restatement of the reference algorithm needs on this workload to reach
# relative KKT 1e-6 (measured by this bench's FP64 leg on a B200; the CPU reference runs the
# same algorithm, so its sample is extrapolated to this count when no GPU leg ran first).
FP64_ITERATIONS_TO_TOLERANCE = 160560
WORKLOAD = ("powerlaw LP 200,000 x 500,000, 5,000,000 nonzeros (10 per column), rows "
            "Pareto(1.5), values N(0,1)*10^U(-2,2) per row, equality rows, 0<=x<=u, planted "
            "optimum, seed 1; relative KKT 1e-6")


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    return world, rank


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(m, n, nnz, value_bytes, algorithm="reference"):
    """Bytes one PDHG attempt must move (A and A' once, the vectors once).

    reference operator: matrix values and int32 indices of both orientations, both
    row-pointer arrays, per column x, c, l, u, the gathered operand and the written x' and
    xbar at the iterate width plus the FP64 running sum, per row y, row bounds, the gathered
    operand and y' plus the FP64 running sum.
    Halpern operator, FP32 level (value_bytes 4): the same matrix terms; per column the delta
    x, c + A'y_r (FP64), the two FP32 relative bounds, the gathered operand, written T(z)_x
    and x_{k+1} (32 B); per row the delta y, y_r, A x_r, both FP64 bounds, the gathered
    operand, written T(z)_y, y_{k+1} and the FP64 A x_{k+1} (56 B). FP64 level: per column x,
    c, l, u, x_0, the gathered operand, T(z)_x, x_{k+1} (64 B); per row y, both bounds, y_0,
    A x_0, the gathered operand, T(z)_y, y_{k+1}, A x_{k+1} (72 B)."""
    s = value_bytes
    matrix = 2 * nnz * (s + 4) + 4 * (m + n + 2)
    if algorithm == "halpern":
        return matrix + (n * 32 + m * 56 if s == 4 else n * 64 + m * 72)
    return matrix + n * (7 * s + 16) + m * (5 * s + 16)


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device=0):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def cpu_reference_sample(lp, iterations):
    """The reference solve_pdhg on the host: setup-only and setup + `iterations` runs."""
    import oracle

    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    if oracle.ref_available():
        kind = "reference"
        run = lambda lim: oracle.ref_solve(lp, tolerance=TOLERANCE, iteration_limit=lim)  # noqa: E731
    else:
        kind = "port"
        threads = 1
        run = lambda lim: oracle.oracle_solve(lp, tolerance=TOLERANCE, iteration_limit=lim)  # noqa: E731
    t0 = time.perf_counter()
    run(0)
    setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    run(iterations)
    with_its = time.perf_counter() - t0
    per_iteration = max(with_its - setup, 1e-9) / iterations
    return kind, threads, setup, per_iteration


CPU_BATCH_CAP = 20000       # iterations charged to an LP the CPU reference cannot certify
CPU_BATCH_PROBE = 200       # iterations timed per LP of the CPU batch sample


def _cpu_worker_init():
    os.environ["OMP_NUM_THREADS"] = "1"


def _cpu_ref_one(args):
    """Setup time and time per iteration of the reference solve_pdhg on one LP (one thread):
    the setup is the faster of two runs without iterations; the iterations are timed over at
    least `probe` of them and at least 10 ms (fewer if the LP converges first)."""
    import oracle

    lp, probe = args

    def run(limit):
        t0 = time.perf_counter()
        r = oracle.ref_solve(lp, tolerance=TOLERANCE, iteration_limit=limit, stop_at_request=True)
        return time.perf_counter() - t0, r.iterations

    setup = min(run(0)[0] for _ in range(2))
    k = probe
    while True:
        t, its = run(k)
        if t - setup >= 0.01 or its < k or k >= 100 * probe:
            break
        k *= 4
    return setup, max(t - setup, 1e-9) / max(1, its)


def cpu_batch_sample(lps, iterations, what="every 8th LP"):
    """The reference solve_pdhg on a sample of the batch, one LP per host core (processes
    started with spawn, OMP_NUM_THREADS=1 each). Each LP is timed for its setup and
    CPU_BATCH_PROBE iterations and charged `iterations[k]` (the reference operator's count on
    the GPU; CPU_BATCH_CAP for an LP the CPU reference cannot certify); the LPs are packed onto
    the cores largest first, and the rate is the sample over that makespan."""
    import multiprocessing as mp

    import oracle

    if not oracle.ref_available():
        return None
    cores = os.cpu_count() or 1
    with mp.get_context("spawn").Pool(cores, initializer=_cpu_worker_init) as pool:
        timed = pool.map(_cpu_ref_one, [(lp, CPU_BATCH_PROBE) for lp in lps], chunksize=1)
    cost = sorted((setup + per_it * its for (setup, per_it), its in zip(timed, iterations)),
                  reverse=True)
    load = [0.0] * cores
    for c in cost:
        load[load.index(min(load))] += c
    makespan = max(load)
    return {"value": len(lps) / makespan, "unit": "LPs/s", "cores": cores, "kind": "reference",
            "seconds": makespan, "cpu_seconds": sum(cost),
            "sample": f"{what} ({len(lps)}), reference solve_pdhg (pdhg_tolerance "
                      f"{TOLERANCE:g}, pdhg_stop_at_request), one process per core "
                      f"(OMP_NUM_THREADS=1): setup and at least {CPU_BATCH_PROBE} iterations (and 10 ms) "
                      f"timed per LP, "
                      f"extrapolated to the iterations the reference operator needed on the GPU "
                      f"(an infeasible LP, which the CPU reference cannot certify, at "
                      f"{CPU_BATCH_CAP}), packed onto the cores largest first"}


def _percentiles(values):
    import numpy as np

    if not values:
        return {"p50": None, "p99": None, "p99.9": None}
    v = np.asarray(values, dtype=np.float64)
    return {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99)),
            "p99.9": float(np.percentile(v, 99.9))}


def batched_leg(local, world, rank, dist, torch, algorithm="halpern"):
    """512 uneven LPs through the batched engine (sharded over ranks), and a one-at-a-time
    FP64 sample on rank 0."""
    from sih26_b200 import lpgen, pdhg
    from sih26_b200.shard import gather_by_index, shard_by_nnz

    lps = lpgen.uneven_batch(count=512, m_lo=50, m_hi=5000, infeasible_fraction=0.1, seed=3)
    mine = shard_by_nnz([lp.num_nonzeros for lp in lps], world)[rank]
    opts = pdhg.Options(pdhg_tolerance=TOLERANCE, pdhg_stop_rule="relative_kkt",
                        gpu_device=local, pdhg_algorithm=algorithm)

    def sync():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    pdhg.batch_solve([lps[k] for k in mine[:64]], opts)  # warm-up (module load, first launch)
    sync()
    t0 = time.perf_counter()
    sols = pdhg.batch_solve([lps[k] for k in mine], opts)
    sync()
    wall = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([wall], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        wall = float(t.item())
    local_out = {}
    for k, s in zip(mine, sols):
        rel = max(s.residuals["relative_primal"], s.residuals["relative_dual"],
                  s.residuals["relative_gap"])
        local_out[k] = (s.status, rel, s.solve_seconds, s.iterations)
    allres = gather_by_index(local_out, dist)
    if rank != 0:
        return None
    planted_infeasible = sum(lp.farkas_star is not None for lp in lps)
    statuses = [allres[k][0] for k in range(len(lps))]
    met = sum(1 for k in range(len(lps)) if lps[k].farkas_star is None
              and statuses[k] in ("optimal", "feasible") and allres[k][1] <= TOLERANCE)
    certified = sum(1 for k in range(len(lps)) if lps[k].farkas_star is not None
                    and statuses[k] == "infeasible")
    # one at a time, plain FP64, on every 8th LP (its feasible ones, and its infeasible ones
    # with the certificate test that the single-LP path also runs)
    sample = list(range(0, len(lps), 8))
    one_rate = one_at_a_time([lps[k] for k in sample], local, algorithm)
    # the reference operator on the same batch, for comparison
    other = "reference" if algorithm == "halpern" else "halpern"
    t0 = time.perf_counter()
    osols = pdhg.batch_solve(lps, pdhg.Options(pdhg_tolerance=TOLERANCE,
                                               pdhg_stop_rule="relative_kkt",
                                               gpu_device=local, pdhg_algorithm=other))
    other_rate = len(lps) / (time.perf_counter() - t0)
    # the reference operator's iteration counts: this batch's when it ran the reference
    # operator, else the comparison batch's
    ref_its = ([osols[k].iterations for k in sample] if other == "reference"
               else [allres[k][3] for k in sample])
    ref_its = [CPU_BATCH_CAP if lps[k].farkas_star is not None else its
               for k, its in zip(sample, ref_its)]
    cpu_batch = cpu_batch_sample([lps[k] for k in sample], ref_its)
    rate = len(lps) / wall
    return {
        "workload": "512 uneven LPs, m log-uniform [50, 5000], n = m U(1.5,3), 5-15 nnz/col, "
                    "10% infeasible, seed 3, relative KKT 1e-6",
        "lps": len(lps), "nonzeros": int(sum(lp.num_nonzeros for lp in lps)),
        "value": rate, "unit": "LPs/s", "seconds": wall,
        "latency_s": _percentiles([allres[k][2] for k in range(len(lps))]),
        "met_tolerance": met, "feasible_lps": len(lps) - planted_infeasible,
        "certified_infeasible": certified, "planted_infeasible": planted_infeasible,
        "precision": "fp64", "algorithm": algorithm,
        f"{other}_operator": {"value": other_rate, "unit": "LPs/s"},
        "one_at_a_time_fp64": {"value": one_rate, "unit": "LPs/s", "algorithm": algorithm,
                               "sample": f"every 8th LP ({len(sample)}), once each"},
        "speedup_vs_one_at_a_time": rate / one_rate,
        "cpu_reference": cpu_batch,
        "sharding": f"{world} rank(s), by nonzeros" if world > 1 else "single GPU",
    }


def served_family(count, seed):
    """The served family: m log-uniform on [100, 50,000], otherwise as the batched one."""
    import math

    import numpy as np

    from sih26_b200 import lpgen

    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        m = int(round(math.exp(rng.uniform(math.log(100), math.log(50000)))))
        n = int(round(m * rng.uniform(1.5, 3.0)))
        out.append(lpgen.small_planted(m, n, 5, 15, rng, name=f"served{k}-{m}x{n}"))
    return out


def one_at_a_time(lps, local, algorithm):
    """LPs/s of the plain FP64 single-LP path, one LP after another (after one warm-up)."""
    from sih26_b200 import pdhg

    one = pdhg.Options(pdhg_tolerance=TOLERANCE, pdhg_stop_rule="relative_kkt",
                       pdhg_precision="fp64", gpu_device=local, pdhg_algorithm=algorithm)
    pdhg.solve_pdhg(lps[0], one)
    t0 = time.perf_counter()
    for lp in lps:
        pdhg.solve_pdhg(lp, one)
    return len(lps) / (time.perf_counter() - t0)


def served_leg(local, rates, seconds, chunk, algorithm="halpern", pool_size=24, seed=5,
               drain_cap=90.0):
    """A Poisson stream at each rate (LPs/s) for `seconds` into a resident server."""
    import concurrent.futures as cf

    import numpy as np

    from sih26_b200 import pdhg

    pool = served_family(pool_size, seed)
    base_rate = one_at_a_time(pool, local, algorithm)
    opts = pdhg.Options(pdhg_tolerance=TOLERANCE, pdhg_stop_rule="relative_kkt",
                        gpu_device=local, pdhg_algorithm=algorithm)
    # the CPU reference on the pool, one LP per host core, charged the iterations the
    # reference operator needs (counted on the GPU)
    ref_sols = pdhg.batch_solve(pool, pdhg.Options(pdhg_tolerance=TOLERANCE,
                                                   pdhg_stop_rule="relative_kkt",
                                                   gpu_device=local,
                                                   pdhg_algorithm="reference"))
    cpu_pool = cpu_batch_sample(pool, [s.iterations for s in ref_sols], "the pool's LPs")
    out = []
    for rate in rates:
        rng = np.random.default_rng(seed + 1)
        arrivals = []
        t = 0.0
        while True:
            t += rng.exponential(1.0 / rate)
            if t > seconds:
                break
            arrivals.append(t)
        picks = rng.integers(0, pool_size, len(arrivals))
        latency, statuses = {}, {}
        with pdhg.Server(device=local, chunk_attempts=chunk) as srv, \
                cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
            srv.solve_all([pool[0]], opts)  # warm-up
            futures, tickets = {}, {}
            nxt = 0
            t0 = time.perf_counter()
            while len(latency) < len(arrivals):
                now = time.perf_counter() - t0
                if now > seconds + drain_cap:
                    break
                while nxt < len(arrivals) and arrivals[nxt] <= now:
                    futures[nxt] = ex.submit(srv.submit, pool[picks[nxt]], opts)
                    nxt += 1
                for k in [k for k, f in futures.items() if f.done()]:
                    tickets[k] = futures.pop(k).result()
                active, waiting, _ = srv.step()
                done_at = time.perf_counter() - t0
                for k in list(tickets):
                    r = srv.result(tickets[k])
                    if r is not None:
                        latency[k] = done_at - arrivals[k]
                        statuses[k] = r.status
                        del tickets[k]
                if active == 0 and waiting == 0 and not tickets:
                    time.sleep(0.0005)
            span = time.perf_counter() - t0
        done = len(latency)
        served_rate = done / span if span > 0 else None
        out.append({
            "workload": f"Poisson arrivals at {rate:g} LPs/s for {seconds:g} s, LPs drawn from "
                        f"a pool of {pool_size} of the served family (m log-uniform [100, "
                        f"50000], n = m U(1.5,3), 5-15 nnz/col, seed {seed}), relative KKT 1e-6",
            "offered_rate": rate, "requests": len(arrivals), "completed": done,
            "optimal_or_feasible": sum(1 for v in statuses.values()
                                       if v in ("optimal", "feasible")),
            "value": served_rate, "unit": "LPs/s", "span_s": span,
            "latency_s": _percentiles(list(latency.values())), "chunk_attempts": chunk,
            "precision": "fp64", "algorithm": algorithm,
            "one_at_a_time_fp64": {"value": base_rate, "unit": "LPs/s",
                                   "sample": f"the {pool_size} LPs of the pool, once each"},
            "speedup_vs_one_at_a_time": (served_rate / base_rate) if served_rate else None,
            "cpu_reference": cpu_pool,
        })
    return out


def qp_leg(local):
    """Convex QP (sankhya_qp_gpu_solve) beside the reference's own QP engine on the host: the
    planted 800 x 2,000 QP (the largest the reference's dense convexity test accepts) to its
    qp_tolerance 1e-6, and a 40,000 x 100,000 one on the GPU alone (convexity asserted by the
    caller, which the reference cannot do)."""
    import oracle
    from sih26_b200 import lpgen, pdhg

    out = {}
    small = lpgen.qp_planted(800, 2000, 10, seed=21)
    big = lpgen.qp_planted(40000, 100000, 10, seed=21)
    for name, lp, assume in (("800x2000", small, False), ("40000x100000", big, True)):
        o = pdhg.Options(qp_tolerance=1e-6, iteration_limit=400000, qp_assume_convex=assume,
                         gpu_device=local)
        pdhg.solve_qp(lp, pdhg.Options(qp_tolerance=1e-6, iteration_limit=100,
                                       qp_assume_convex=assume, gpu_device=local))
        t0 = time.perf_counter()
        s = pdhg.solve_qp(lp, o)
        gpu = time.perf_counter() - t0
        rec = {"gpu_s": gpu, "status": s.status, "iterations": s.iterations,
               "objective_rel_error": abs(s.objective - lp.optimal_objective)
               / abs(lp.optimal_objective)}
        if not assume and oracle.ref_available():
            t0 = time.perf_counter()
            r = oracle.ref_qp_solve(lp, tolerance=1e-6, iteration_limit=400000)
            rec["reference_s"] = time.perf_counter() - t0
            rec["reference_iterations"] = r.iterations
            rec["reference_status"] = r.status
        out[name] = rec
    return out


def make_workload():
    from sih26_b200 import lpgen

    return lpgen.powerlaw_planted(seed=SEED)


def run_reference(args):
    world, rank = _dist()
    if rank != 0:
        return 0
    lp = make_workload()
    values = []
    info = None
    for step in range(args.warmup + args.steps):
        kind, threads, setup, per_it = cpu_reference_sample(lp, REF_SAMPLE_ITERATIONS)
        est = setup + per_it * FP64_ITERATIONS_TO_TOLERANCE
        if step >= args.warmup:
            values.append(est)
            info = (kind, threads, setup, per_it)
    kind, threads, setup, per_it = info
    value = statistics.mean(values)
    sample = (f"solve_pdhg setup ({setup:.2f} s) + {REF_SAMPLE_ITERATIONS} iterations "
              f"({per_it * 1e3:.2f} ms each) per step, extrapolated to "
              f"{FP64_ITERATIONS_TO_TOLERANCE} iterations")
    line = {
        "impl": "reference", "metric": "time-to-rel-KKT 1e-6 (s)", "value": value, "unit": "s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD},
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch

    from sih26_b200 import pdhg

    world, rank = _dist()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    lp = make_workload()
    m, n, nnz = lp.num_rows, lp.num_cols, lp.num_nonzeros
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def opts(precision, algorithm, profile=False):
        # the autotuner measures the schedules in the first warm-up solve and caches them
        return pdhg.Options(pdhg_tolerance=TOLERANCE, pdhg_stop_rule="relative_kkt",
                            pdhg_precision=precision, pdhg_algorithm=algorithm,
                            gpu_device=local, pdhg_profile_kernels=profile,
                            pdhg_autotune=True)

    def sync():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def step(precision, algorithm, profile=False):
        flush.random_(0, 255)  # L2 flush between steps
        sync()
        s = pdhg.solve_pdhg(lp, opts(precision, algorithm, profile))
        sync()
        return s

    algo = args.algorithm
    other = "reference" if algo == "halpern" else "halpern"
    for _ in range(args.warmup):
        step("mixed", algo)
    sols = []
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            sols.append(step("mixed", algo, profile=True))
    fp64 = step("fp64", algo)
    alt_mixed = step("mixed", other)
    alt_fp64 = step("fp64", other)

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    dev = max_over_ranks(statistics.mean(s.device_seconds for s in sols))
    e2e = max_over_ranks(statistics.mean(s.solve_seconds for s in sols))
    fp64_dev = max_over_ranks(fp64.device_seconds)
    alt = {k: {"value": max_over_ranks(v.device_seconds), "unit": "s",
               "iterations": v.iterations, "status": v.status}
           for k, v in (("mixed", alt_mixed), ("fp64", alt_fp64))}
    last = sols[-1]
    for s in sols:
        if s.status not in ("optimal", "feasible"):
            raise SystemExit(f"solve did not converge: {s.status} {s.message}")
        rel = max(s.residuals["relative_primal"], s.residuals["relative_dual"],
                  s.residuals["relative_gap"])
        if rel > TOLERANCE:
            raise SystemExit(f"solve stopped above the tolerance: {rel}")
    # roofline of the iteration kernel: attempts are all FP32 unless the polish ran
    attempts = sum(s.attempts for s in sols)
    kern = sum(s.iterate_kernel_seconds for s in sols)
    fp32_share = sum(s.fp32_iterations for s in sols) / max(1, sum(s.iterations for s in sols))
    bytes_attempt = (fp32_share * algorithmic_bytes(m, n, nnz, 4, algo)
                     + (1 - fp32_share) * algorithmic_bytes(m, n, nnz, 8, algo))
    achieved = bytes_attempt * attempts / kern / 1e9 if kern > 0 else None
    peak, peak_kind = _peaks()
    traffic = None
    summary = os.path.join(ROOT, "profiles", "iterate_kernel_powerlaw_200k.md")
    if os.path.exists(summary):
        for line in open(summary):
            if line.startswith("dram_bytes_per_attempt:"):
                traffic = float(line.split(":")[1].strip().split()[0])
    cpu = None
    if rank == 0:
        kind, threads, setup, per_it = cpu_reference_sample(lp, REF_SAMPLE_ITERATIONS)
        cpu = {"value": setup + per_it * fp64.iterations, "unit": "s", "cores": threads,
               "kind": kind,
               "sample": (f"solve_pdhg setup ({setup:.2f} s) + {REF_SAMPLE_ITERATIONS} "
                          f"iterations ({per_it * 1e3:.2f} ms each), extrapolated to the "
                          f"{fp64.iterations} iterations the FP64 GPU leg needed")}
    launches = int(statistics.mean(s.kernel_launches for s in sols))
    batched = (None if args.no_batched
               else batched_leg(local, world, rank, dist, torch, args.algorithm))
    served = None
    if rank == 0 and not args.no_served:
        rates = [float(r) for r in args.served_rates.split(",") if r]
        served = served_leg(local, rates, args.served_seconds, args.served_chunk,
                            args.algorithm)
    qp = qp_leg(local) if rank == 0 and not args.no_qp else None
    if rank == 0:
        line = {
            "metric": "time-to-rel-KKT 1e-6 (s), FP32-mixed", "value": dev, "unit": "s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 iterates, f64 reductions",
            "data": "synthetic (seeded planted-optimum LP)",
            "config": {"workload": WORKLOAD, "tolerance": TOLERANCE,
                       "stop_rule": "relative_kkt", "precision": "mixed", "algorithm": algo,
                       "l2": "inputs larger than L2 (A, A' and vectors ~0.3 GB resident) and a "
                             "256 MB L2 flush before every step",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "iterations": last.iterations, "fp32_iterations": last.fp32_iterations,
            "schedule": {"autotuned": last.autotuned, "stream_row_max_A": last.schedule[0],
                         "nnz_per_lane_A": last.schedule[1],
                         "stream_row_max_AT": last.schedule[2],
                         "nnz_per_lane_AT": last.schedule[3]},
            "attempts": last.attempts, "restarts": last.restarts,
            "objective_rel_error": abs(last.objective - lp.optimal_objective)
            / abs(lp.optimal_objective),
            "fp64": {"value": fp64_dev, "unit": "s", "iterations": fp64.iterations,
                     "status": fp64.status},
            "algorithm": algo,
            f"{other}_operator": alt,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "iterate_kernel",
                         "bytes_per_attempt": bytes_attempt,
                         "us_per_attempt": kern / attempts * 1e6 if attempts else None},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": last.h2d_bytes,
                    "d2h_bytes_per_step": last.d2h_bytes,
                    "setup_s": statistics.mean(s.setup_seconds for s in sols)},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "batched": batched,
            "served": served,
            "qp": qp,
        }
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def profile_run(kind, algorithm):
    """Bounded runs for ncu captures (no timing, no JSON): `single` runs the 5M-nonzero LP for
    200 iterations in FP32-mixed and again in FP64; `batch` solves the first 64 LPs of the
    batched family in one batched call; both with the operator of --algorithm."""
    from sih26_b200 import lpgen, pdhg

    if kind == "single":
        lp = make_workload()
        for precision in ("mixed", "fp64"):
            s = pdhg.solve_pdhg(lp, pdhg.Options(pdhg_tolerance=TOLERANCE, iteration_limit=200,
                                                 pdhg_stop_rule="relative_kkt",
                                                 pdhg_precision=precision,
                                                 pdhg_algorithm=algorithm))
            print(precision, s.status, s.iterations, s.kernel_launches)
    else:
        lps = lpgen.uneven_batch(count=512, m_lo=50, m_hi=5000, infeasible_fraction=0.1, seed=3)
        sols = pdhg.batch_solve(lps[:64], pdhg.Options(pdhg_tolerance=TOLERANCE,
                                                       pdhg_stop_rule="relative_kkt",
                                                       pdhg_algorithm=algorithm))
        print("batch", sum(s.status in ("optimal", "feasible", "infeasible") for s in sols))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--algorithm", choices=["halpern", "reference"], default="halpern",
                    help="iteration operator of the timed solves (the other one is timed once "
                         "in each precision for comparison)")
    ap.add_argument("--no-batched", action="store_true", help="skip the 512-LP batched leg")
    ap.add_argument("--no-served", action="store_true", help="skip the served-stream leg")
    ap.add_argument("--no-qp", action="store_true", help="skip the convex-QP leg")
    ap.add_argument("--served-rates", default="50,200",
                    help="Poisson rates, LPs/s, comma-separated (the served family's full "
                         "study is 200,1000,5000 for 60 s)")
    ap.add_argument("--served-seconds", type=float, default=4.0, help="arrival window, s")
    ap.add_argument("--served-chunk", type=int, default=512,
                    help="attempts per LP per server launch")
    ap.add_argument("--profile-run", choices=["single", "batch"], default=None,
                    help="a bounded run for an ncu capture (prints no bench line)")
    args = ap.parse_args()
    if args.profile_run:
        return profile_run(args.profile_run, args.algorithm)
    if args.warmup < 3:
        raise SystemExit("at least 3 warm-up steps")
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
