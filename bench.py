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
          threads, on a bounded sample: setup + 20 iterations, extrapolated to the iterations
          the reference's operator needs in FP64 (counted by this run's FP64 reference-operator
          leg on the GPU)

  batched  512 uneven LPs (m log-uniform on [50, 5,000], n = m U(1.5, 3), 5-15 nonzeros per
          column, 10 % primal-infeasible; lpgen.uneven_batch, seed 3) solved to relative KKT
          1e-6 by the batched engine in one call (sankhya_pdhg_gpu_batch_solve, host arrays in
          and out): LPs/s, p50 / p99 / p99.9 submit-to-answer latency, certificates found, and
          the same LPs solved one at a time by the plain FP64 single-LP path (a sample of every
          8th LP) for the LPs/s ratio. Under torchrun the 512 LPs are sharded by nonzeros
          (sih26_b200.shard) and the time is the maximum over ranks.
  served  Poisson request streams at 200, 1,000 and 5,000 LPs/s for 20 s each (--served-seconds 60
          for the survey's full windows), every request a fresh LP of the served family (m
          log-uniform on [100, 50,000], 10 % infeasible; lpgen.served_request), into a resident
          server that admits requests between launches of its persistent kernels (continuous
          batching): LPs/s and p50 / p99 / p99.9 arrival-to-answer latency, per size class too,
          next to one-at-a-time FP64 solves of the stream's first LPs. Rank 0 only.
  configs the 2,000 x 5,000 LP (with the reference CPU solver run to tolerance for real), the
          headline LP at 1e-4 and 1e-8, and the 258,000 x 640,000 block-angular LP, each answer
          checked by the oracle (see config_legs).
  parity  the headline answer's residuals recomputed by the oracle from the returned point, and
          its active-bound pattern against the planted optimum (see parity_of).

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
METRIC = "time-to-rel-KKT 1e-6 (s)"
REF_SAMPLE_ITERATIONS = 20
# Iterations the reference's own operator needs on this workload to reach relative KKT 1e-6 in
# FP64: 167,280, measured by this bench's FP64 reference-operator leg on a B200 (that leg runs
# the reference's algorithm, src/pdhg/pdhg.cpp:383-644, in FP64; the CPU reference cannot be
# run to tolerance here, it would take over an hour). The reference arm extrapolates its timed
# sample to this count; the main arm uses the count its own FP64 reference-operator leg
# measured in the same run.
FP64_ITERATIONS_TO_TOLERANCE = 167280
# DRAM bytes per step of the FP32 Halpern iteration kernel on this workload, from one ncu
# capture of a 40-step launch (dram__bytes_read.sum + dram__bytes_write.sum = 1.620 + 0.032 GB
# over 40 steps; captured with `ncu --set full --clock-control none --kernel-name-base demangled
# -k regex:"iterate_kernel<float" -s 1 -c 1 python bench.py --profile-run single`). Recaptured
# whenever the kernel changes.
ITERATE_DRAM_BYTES_PER_STEP = 41.3e6
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
    one_rate, _ = one_at_a_time([lps[k] for k in sample], local, algorithm)
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


def _gen_request(args):
    """One request of the served stream (runs in a generator process)."""
    seed, index = args
    from sih26_b200 import lpgen

    return lpgen.served_request(index, seed)


def _size_class(m):
    return "m<1000" if m < 1000 else ("m<10000" if m < 10000 else "m>=10000")


def one_at_a_time(lps, local, algorithm):
    """LPs/s of the plain FP64 single-LP path, one LP after another (after one warm-up; the
    faster of two passes), and the seconds each LP took."""
    from sih26_b200 import pdhg

    one = pdhg.Options(pdhg_tolerance=TOLERANCE, pdhg_stop_rule="relative_kkt",
                       pdhg_precision="fp64", gpu_device=local, pdhg_algorithm=algorithm)
    pdhg.solve_pdhg(lps[0], one)
    best = None
    for _ in range(2):  # the faster of two passes: the host's load varies between them
        each = []
        t0 = time.perf_counter()
        for lp in lps:
            t1 = time.perf_counter()
            pdhg.solve_pdhg(lp, one)
            each.append(time.perf_counter() - t1)
        total = time.perf_counter() - t0
        if best is None or total < best[0]:
            best = (total, each)
    return len(lps) / best[0], best[1]


def served_leg(local, rates, seconds, chunk, algorithm="halpern", seed=5, drain_cap=15.0,
               sample=64, max_active=1024, backlog=64, workers=8, solo_min_nnz=0):
    """Poisson request streams at each rate (LPs/s) for `seconds` into a resident server.

    Every request is a fresh LP (lpgen.served_request: m log-uniform on [100, 50,000],
    n = m U(1.5, 3), 5-15 nonzeros per column, 10 % primal-infeasible), drawn by a pool of
    generator processes ahead of need; a request's content exists when it arrives, so drawing
    it is not part of its latency. The client hands the server the oldest arrived request
    whenever fewer than `backlog` wait inside it (host preparation runs on the submitting
    threads); the server admits waiting LPs between launches as slots (`max_active`) and pool
    memory (80 % of free HBM) allow, and every active LP advances in every launch (continuous
    batching). Latency is arrival to verified answer. Requests still unanswered `drain_cap`
    seconds after the window closes are reported as unfinished, and the latency percentiles
    then count them at their age (lower bounds)."""
    import collections
    import concurrent.futures as cf
    import multiprocessing as mp

    import numpy as np

    from sih26_b200 import pdhg

    opts = pdhg.Options(pdhg_tolerance=TOLERANCE, pdhg_stop_rule="relative_kkt",
                        gpu_device=local, pdhg_algorithm=algorithm)
    gen = cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn"))
    try:
        base = list(gen.map(_gen_request, [(seed, k) for k in range(sample)]))
        base_rate, base_each = one_at_a_time(base, local, algorithm)
        by_class_one = collections.defaultdict(list)
        for lp, t in zip(base, base_each):
            by_class_one[_size_class(lp.num_rows)].append(t)
        # the CPU reference on part of the sample, one LP per host core, charged the
        # iterations the reference operator needs (counted on the GPU)
        cpu_lps = base[:16]
        ref_sols = pdhg.batch_solve(cpu_lps, pdhg.Options(
            pdhg_tolerance=TOLERANCE, pdhg_stop_rule="relative_kkt", gpu_device=local,
            pdhg_algorithm="reference"))
        ref_its = [CPU_BATCH_CAP if lp.farkas_star is not None else r.iterations
                   for lp, r in zip(cpu_lps, ref_sols)]
        cpu_pool = cpu_batch_sample(cpu_lps, ref_its, "the stream's first LPs")
        out = []
        for rate in rates:
            rseed = seed * 1000 + int(rate)
            rng = np.random.default_rng(rseed)
            arrivals = []
            t = 0.0
            while True:
                t += rng.exponential(1.0 / rate)
                if t > seconds:
                    break
                arrivals.append(t)
            N = len(arrivals)
            ahead = 256
            gen_f, sub_f, tickets = {}, {}, {}
            latency, status, kkt, size = {}, {}, {}, {}
            next_gen = next_sub = 0
            with pdhg.Server(device=local, chunk_attempts=chunk, max_active=max_active,
                             solo_min_nnz=solo_min_nnz) as srv, \
                    cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
                srv.solve_all([base[0]], opts)  # warm-up
                waiting = 0
                t0 = time.perf_counter()
                while True:
                    now = time.perf_counter() - t0
                    if now > seconds + drain_cap:
                        break
                    arrived = int(np.searchsorted(arrivals, now, side="right"))
                    if now > seconds and len(latency) >= arrived:
                        break
                    while next_gen < N and next_gen - next_sub < ahead:
                        gen_f[next_gen] = gen.submit(_gen_request, (rseed, next_gen))
                        next_gen += 1
                    while (next_sub < arrived and waiting + len(sub_f) < backlog
                           and gen_f[next_sub].done()):
                        lp = gen_f.pop(next_sub).result()
                        size[next_sub] = lp.num_rows
                        sub_f[next_sub] = ex.submit(srv.submit, lp, opts)
                        next_sub += 1
                    for k in [k for k, f in sub_f.items() if f.done()]:
                        tickets[k] = sub_f.pop(k).result()
                    active, waiting, _ = srv.step()
                    done_at = time.perf_counter() - t0
                    for k in list(tickets):
                        r = srv.result(tickets[k])
                        if r is not None:
                            latency[k] = done_at - arrivals[k]
                            status[k] = r.status
                            kkt[k] = _rel_kkt(r) if r.residuals else None
                            del tickets[k]
                    if active == 0 and waiting == 0 and not tickets and not sub_f:
                        time.sleep(0.0005)
                span = time.perf_counter() - t0
                launch_settings = srv.stats()
                for f in sub_f.values():
                    f.result()
            for f in gen_f.values():
                f.cancel()
            unfinished = [k for k in range(N) if k not in latency]
            ages = list(latency.values()) + [span - arrivals[k] for k in unfinished]
            feasible_ok = sum(1 for k, v in status.items()
                              if v in ("optimal", "feasible") and kkt[k] is not None
                              and kkt[k] <= TOLERANCE)
            classes = {}
            for cname in ("m<1000", "m<10000", "m>=10000"):
                ks = [k for k in latency if _size_class(size[k]) == cname]
                one = by_class_one.get(cname, [])
                classes[cname] = {
                    "completed": len(ks), "value": len(ks) / span if span > 0 else None,
                    "latency_s": _percentiles([latency[k] for k in ks]),
                    "one_at_a_time_s_per_lp": (sum(one) / len(one)) if one else None}
            served_rate = len(latency) / span if span > 0 else None
            out.append({
                "workload": f"Poisson arrivals at {rate:g} LPs/s for {seconds:g} s, every "
                            f"request a fresh LP (m log-uniform [100, 50000], n = m U(1.5,3), "
                            f"5-15 nnz/col, 10% infeasible), relative KKT 1e-6",
                "offered_rate": rate, "seconds": seconds, "requests": N,
                "completed": len(latency), "unfinished": len(unfinished),
                "optimal_or_feasible": feasible_ok,
                "certified_infeasible": sum(1 for v in status.values() if v == "infeasible"),
                "value": served_rate, "unit": "LPs/s", "span_s": span,
                "latency_s": _percentiles(ages), "latency_censored": bool(unfinished),
                "chunk_attempts": chunk, "max_active": max_active, "solo_min_nnz": solo_min_nnz,
                "launch_settings": launch_settings,
                "precision": "fp64", "algorithm": algorithm,
                "one_at_a_time_fp64": base_rate,
                "speedup_vs_one_at_a_time": (served_rate / base_rate) if served_rate else None,
                "by_size": classes,
                "cpu_reference": cpu_pool,
            })
        return out
    finally:
        gen.shutdown(wait=False, cancel_futures=True)


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


def parity_of(lp, s):
    """Parity of a returned answer, checked on the host after the timed region: the oracle's
    unscaled residuals of the point (two FP64 SpMVs of the C restatement of the reference's
    evaluate(), src/pdhg/pdhg.cpp:143-263, from x and row_dual alone), and its active-bound
    pattern on the columns whose planted reduced cost is nonzero. The planted optimum is
    strictly complementary (|z| >= 0.1), so every optimal point has those columns at the
    planted bound; the other columns may sit anywhere on the optimal face."""
    import numpy as np

    import oracle

    sense = -1.0 if lp.maximize else 1.0
    r = oracle.oracle_evaluate(lp, s.col_value, -sense * s.row_dual)
    out = {"rel_kkt_oracle": max(r["primal"], r["dual"], r["gap"]),
           "rel_primal": r["primal"], "rel_dual": r["dual"], "rel_gap": r["gap"],
           "status": s.status}
    if lp.x_star is not None and lp.row_dual_star is not None:
        z = lp.cost - lp.to_scipy_csc().T @ lp.row_dual_star
        x = s.col_value
        lo, hi = lp.col_lower, lp.col_upper
        at_lo = np.abs(x - lo) <= 1e-6 * np.maximum(1.0, np.abs(lo))
        at_hi = np.abs(x - hi) <= 1e-6 * np.maximum(1.0, np.abs(hi))
        forced_lo, forced_hi = z > 0.05, z < -0.05
        out["pattern_checked_columns"] = int(forced_lo.sum() + forced_hi.sum())
        out["pattern_mismatches"] = int((forced_lo & ~at_lo).sum() + (forced_hi & ~at_hi).sum())
        out["objective_rel_error"] = (abs(s.objective - lp.optimal_objective)
                                      / max(1.0, abs(lp.optimal_objective)))
    return out


def _rel_kkt(s):
    r = s.residuals
    return max(r["relative_primal"], r["relative_dual"], r["relative_gap"])


def config_legs(local, flush, sync, fp64_ref_iterations):
    """The other single-LP configurations, each solved once outside the timed region, through
    the C ABI from host arrays, with its answer checked by the oracle:

      c0  2,000 x 5,000 uniform LP (lpgen.uniform_planted, seed 0), relative KKT 1e-6: the GPU
          (FP64 with the reference's operator, and FP32-mixed Halpern) next to the reference's
          own solve_pdhg run to the same tolerance on all host threads, for real;
      c1  the headline LP at relative KKT 1e-4 and 1e-8 (FP32-mixed Halpern; the FP64 polish
          takes over when the FP32 level stops improving), and at 1e-8 with the hand-over to
          the FP64 polish forced at 1e-6;
      c2  the block-angular LP (64 blocks of 4,000 x 10,000, 8 nonzeros per column, 2,000
          linking rows over 2 % of the columns, 30 % '<=' rows; lpgen.block_angular_planted,
          seed 2, 258,000 x 640,000, 30.7M nonzeros), FP32-mixed Halpern to 1e-6, with the
          roofline of its iteration kernel."""
    import oracle
    from sih26_b200 import lpgen, pdhg

    peak, _ = _peaks()
    out = {}

    def solve(lp, tol, precision, algorithm, profile=False, switch=0.0):
        flush.random_(0, 255)
        sync()
        s = pdhg.solve_pdhg(lp, pdhg.Options(
            pdhg_tolerance=tol, pdhg_stop_rule="relative_kkt", pdhg_precision=precision,
            pdhg_algorithm=algorithm, gpu_device=local, pdhg_profile_kernels=profile,
            pdhg_autotune=True, pdhg_mixed_switch_tolerance=switch))
        sync()
        return s

    def record(lp, s, tol):
        p = parity_of(lp, s)
        return {"device_s": s.device_seconds, "e2e_s": s.solve_seconds,
                "iterations": s.iterations, "fp32_iterations": s.fp32_iterations,
                "rel_kkt": _rel_kkt(s), "tolerance": tol, **p}

    # c0: small enough for the CPU reference to run to tolerance. Its GPU solves last ~10-20 ms,
    # where host jitter shows, so each keeps the faster of two (same answer both times).
    lp0 = lpgen.uniform_planted(2000, 5000, 10, seed=0)
    solve(lp0, TOLERANCE, "fp64", "reference")  # warm-up of this shape

    def best_of_two(precision, algorithm):
        a = solve(lp0, TOLERANCE, precision, algorithm)
        b = solve(lp0, TOLERANCE, precision, algorithm)
        return a if a.solve_seconds <= b.solve_seconds else b

    c0 = {"fp64_reference_operator": record(lp0, best_of_two("fp64", "reference"), TOLERANCE),
          "mixed_halpern": record(lp0, best_of_two("mixed", "halpern"), TOLERANCE)}
    if oracle.ref_available():
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        oracle.ref_solve(lp0, tolerance=TOLERANCE, iteration_limit=50, stop_at_request=True)
        t0 = time.perf_counter()
        r = oracle.ref_solve(lp0, tolerance=TOLERANCE, stop_at_request=True)
        cpu_s = time.perf_counter() - t0
        pr = parity_of(lp0, r)
        c0["cpu_reference"] = {"seconds": cpu_s, "iterations": r.iterations,
                               "status": r.status, "threads": int(os.environ["OMP_NUM_THREADS"]),
                               "kind": "reference, run to tolerance (pdhg_stop_at_request)",
                               "rel_kkt_oracle": pr["rel_kkt_oracle"],
                               "pattern_mismatches": pr.get("pattern_mismatches")}
        c0["cpu_over_gpu_e2e"] = cpu_s / c0["fp64_reference_operator"]["e2e_s"]
    out["c0"] = c0

    # c1 at the survey's other tolerances
    lp1 = make_workload()
    for tol in (1e-4, 1e-8):
        out[f"c1_{tol:g}"] = record(lp1, solve(lp1, tol, "mixed", "halpern"), tol)
    # the anchored FP32 level reaches 1e-8 by itself; with the hand-over forced at 1e-6 the FP64
    # polish finishes the solve, for comparison
    out["c1_1e-08_polish_from_1e-06"] = record(lp1, solve(lp1, 1e-8, "mixed", "halpern",
                                                          switch=1e-6), 1e-8)
    del lp1

    # c2: the block-angular LP
    lp2 = lpgen.block_angular_planted()
    solve(lp2, 1e-2, "mixed", "halpern")  # warm-up and autotune of this shape
    s2 = solve(lp2, TOLERANCE, "mixed", "halpern", profile=True)
    c2 = record(lp2, s2, TOLERANCE)
    share = s2.fp32_iterations / max(1, s2.iterations)
    m, n, nnz = lp2.num_rows, lp2.num_cols, lp2.num_nonzeros
    b = (share * algorithmic_bytes(m, n, nnz, 4, "halpern")
         + (1 - share) * algorithmic_bytes(m, n, nnz, 8, "halpern"))
    if s2.iterate_kernel_seconds > 0:
        ach = b * s2.attempts / s2.iterate_kernel_seconds / 1e9
        c2["roofline"] = {"achieved": ach, "peak": peak, "frac": ach / peak,
                          "bytes_per_attempt": b,
                          "us_per_attempt": s2.iterate_kernel_seconds / s2.attempts * 1e6}
    out["c2"] = c2
    out["fp64_reference_operator_iterations_c1"] = fp64_ref_iterations
    return out


def run_reference(args):
    """The reference arm: the reference's own solve_pdhg (oracle/_ref, built from its sources)
    on the host cores. A step is a bounded sample of the headline solve (setup + 20 iterations)
    extrapolated to FP64_ITERATIONS_TO_TOLERANCE; the 2,000 x 5,000 LP is also run to
    tolerance for real once."""
    world, rank = _dist()
    if rank != 0:
        return 0
    import oracle
    from sih26_b200 import lpgen

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
    c0 = None
    if oracle.ref_available():
        lp0 = lpgen.uniform_planted(2000, 5000, 10, seed=0)
        t0 = time.perf_counter()
        r = oracle.ref_solve(lp0, tolerance=TOLERANCE, stop_at_request=True)
        c0 = {"seconds": time.perf_counter() - t0, "iterations": r.iterations,
              "status": r.status, "kind": "reference, run to tolerance"}
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": "fp64", "algorithm": "reference"},
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": kind,
                         "extrapolated": True,
                         "iterations_charged": FP64_ITERATIONS_TO_TOLERANCE,
                         "sample": f"setup {setup:.2f} s + {REF_SAMPLE_ITERATIONS} its at "
                                   f"{per_it * 1e3:.2f} ms, extrapolated"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "c0_to_tolerance": c0,
    }
    print(json.dumps(line))
    return 0


def _brief_batched(b):
    """The batched leg's headline figures, early in the line."""
    if not b:
        return None
    lat = b["latency_s"]
    return {"value": b["value"], "unit": "LPs/s", "p50_s": lat["p50"], "p99_s": lat["p99"],
            "p99.9_s": lat["p99.9"], "met_tolerance": b["met_tolerance"],
            "feasible_lps": b["feasible_lps"], "certified_infeasible": b["certified_infeasible"],
            "planted_infeasible": b["planted_infeasible"],
            "one_at_a_time_fp64": b["one_at_a_time_fp64"]["value"],
            "speedup_vs_one_at_a_time": b["speedup_vs_one_at_a_time"],
            "cpu_reference": (b["cpu_reference"] or {}).get("value")}


def _brief_served(v):
    lat = v["latency_s"]
    keep = ("offered_rate", "seconds", "requests", "completed", "optimal_or_feasible",
            "certified_infeasible", "value", "unfinished", "speedup_vs_one_at_a_time",
            "one_at_a_time_fp64", "chunk_attempts", "launch_settings", "by_size")
    out = {k: v[k] for k in keep if k in v}
    out.update({"p50_s": lat["p50"], "p99_s": lat["p99"], "p99.9_s": lat["p99.9"],
                "latency_censored": v.get("latency_censored"),
                "cpu_reference": (v.get("cpu_reference") or {}).get("value")})
    return out


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
        if _rel_kkt(s) > TOLERANCE:
            raise SystemExit(f"solve stopped above the tolerance: {_rel_kkt(s)}")
    # roofline of the iteration kernel: attempts are all FP32 unless the polish ran
    attempts = sum(s.attempts for s in sols)
    kern = sum(s.iterate_kernel_seconds for s in sols)
    fp32_share = sum(s.fp32_iterations for s in sols) / max(1, sum(s.iterations for s in sols))
    bytes_attempt = (fp32_share * algorithmic_bytes(m, n, nnz, 4, algo)
                     + (1 - fp32_share) * algorithmic_bytes(m, n, nnz, 8, algo))
    achieved = bytes_attempt * attempts / kern / 1e9 if kern > 0 else None
    peak, peak_kind = _peaks()
    traffic = ITERATE_DRAM_BYTES_PER_STEP if algo == "halpern" else None
    # the reference's own operator in FP64 is what the CPU reference runs: its iteration count
    # on this GPU is the count both CPU figures are charged
    ref_its = alt_fp64.iterations if algo == "halpern" else fp64.iterations
    cpu = None
    parity = None
    if rank == 0:
        kind, threads, setup, per_it = cpu_reference_sample(lp, REF_SAMPLE_ITERATIONS)
        cpu = {"value": setup + per_it * ref_its, "unit": "s", "cores": threads, "kind": kind,
               "extrapolated": True, "iterations_charged": ref_its,
               "sample": f"setup {setup:.2f} s + {REF_SAMPLE_ITERATIONS} its at "
                         f"{per_it * 1e3:.2f} ms, extrapolated"}
        parity = parity_of(lp, last)
    launches = int(statistics.mean(s.kernel_launches for s in sols))
    configs = None
    if rank == 0 and not args.no_configs:
        configs = config_legs(local, flush, sync, ref_its)
    batched = (None if args.no_batched
               else batched_leg(local, world, rank, dist, torch, args.algorithm))
    served = None
    if rank == 0 and not args.no_served:
        rates = [float(r) for r in args.served_rates.split(",") if r]
        served = served_leg(local, rates, args.served_seconds, args.served_chunk,
                            args.algorithm, max_active=args.served_max_active,
                            solo_min_nnz=args.served_solo_nnz)
    qp = qp_leg(local) if rank == 0 and not args.no_qp else None
    if rank == 0:
        line = {
            "metric": METRIC, "value": dev, "unit": "s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 iterates, f64 reductions",
            "data": "synthetic (seeded planted-optimum LP)",
            "gpu_launches": launches,
            "config": {"workload": WORKLOAD, "tolerance": TOLERANCE,
                       "stop_rule": "relative_kkt", "precision": "mixed", "algorithm": algo,
                       "l2": "inputs larger than L2 (A, A' and vectors ~0.3 GB resident) and a "
                             "256 MB L2 flush before every step",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "e2e": {"value": e2e, "unit": "s", "h2d_bytes_per_step": last.h2d_bytes,
                    "d2h_bytes_per_step": last.d2h_bytes,
                    "setup_s": statistics.mean(s.setup_seconds for s in sols)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "iterate_kernel",
                         "bytes_per_attempt": bytes_attempt,
                         "us_per_attempt": kern / attempts * 1e6 if attempts else None},
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "parity": parity,
            "fp64": {"value": fp64_dev, "unit": "s", "iterations": fp64.iterations,
                     "status": fp64.status},
            "iterations": last.iterations, "fp32_iterations": last.fp32_iterations,
            "attempts": last.attempts, "restarts": last.restarts,
            "algorithm": algo,
            f"{other}_operator": alt,
            "schedule": {"autotuned": last.autotuned, "A": list(last.schedule[:2]),
                         "AT": list(last.schedule[2:])},
            "batched": _brief_batched(batched),
            "served": [_brief_served(v) for v in served] if served else None,
            "configs": configs,
            "qp": qp,
            "batched_detail": batched,
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
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the 2,000 x 5,000, block-angular and 1e-4 / 1e-8 legs")
    ap.add_argument("--served-rates", default="200,1000,5000",
                    help="Poisson rates, LPs/s, comma-separated")
    ap.add_argument("--served-seconds", type=float, default=20.0,
                    help="arrival window per rate, s (the survey's study is 60)")
    ap.add_argument("--served-chunk", type=int, default=-1,
                    help="attempts per LP per server launch (-1, the default: the server's "
                         "autotuner)")
    ap.add_argument("--served-max-active", type=int, default=1024,
                    help="LP slots of the server in the served leg")
    ap.add_argument("--served-solo-nnz", type=int, default=0,
                    help="served LPs from this many nonzeros go to the single-LP engine (0: never)")
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
