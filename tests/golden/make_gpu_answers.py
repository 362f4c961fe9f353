"""Makes tests/golden/gpu_answers/: answers of the GPU engine, written as the reference's
files (a model .mps.gz and a .sol.gz per case, tests/sol_io.py), for the reference's
independent verifier tools/verify_solution.py to judge (tests/test_verify_gpu_answers.py
runs it where the reference tree exists). Run on a GPU box:

    python tests/golden/make_gpu_answers.py <output directory>

and copy the directory's files into tests/golden/gpu_answers/. The cases (``cases()``) are
the parity LPs (the reference's unit-test LPs, LPs with every row and bound kind, planted
instances, the Netlib LPs of the reference tree), infeasible and unbounded LPs with their
certificates, and a sample of the batched family solved through the batched engine, 10 %
of them infeasible. Every solve uses the reference's stop rule, so `optimal` carries the
reference's meaning (the project's absolute standard holds).
"""
import gzip
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def cases():
    """[(name, lp, how)] with how one of 'fp64', 'mixed', 'halpern', 'batch'."""
    from sih26_b200 import lpgen
    from tests.cases import generated_cases, hand_cases, netlib_cases
    from tests.test_quality_oracle import edge_lps

    out = []
    for name, lp, _ in hand_cases():
        out.append((f"hand_{name}", lp, "fp64"))
    for name, lp in edge_lps():
        out.append((name, lp, "fp64"))
    for name, lp in generated_cases():
        out.append((f"{name}_fp64", lp, "fp64"))
        out.append((f"{name}_mixed", lp, "mixed"))
    for lp, _, _, _ in netlib_cases():
        out.append((f"netlib_{lp.name}", lp, "halpern"))
    rng = np.random.default_rng(41)
    out.append(("infeasible_hand", lpgen.from_dense([[1, 1]], [3], [3], [1, 1],
                                                    col_upper=[1.0, 1.0], name="infeasible_hand"),
                "fp64"))
    for seed in (1, 2):
        base = lpgen.uniform_planted(60, 150, 4, seed=seed)
        out.append((f"infeasible_{seed}", lpgen.make_infeasible(base, rng), "fp64"))
        out.append((f"unbounded_{seed}", lpgen.make_unbounded(base, rng), "fp64"))
    batch = lpgen.uneven_batch(count=40, m_lo=50, m_hi=200, infeasible_fraction=0.1, seed=8)
    for k, lp in enumerate(batch):
        out.append((f"batch_{k:02d}", lp, "batch"))
    return out


def solve_all(cs):
    """The GPU answers of every case, in order."""
    from sih26_b200 import pdhg as P

    opts = {"fp64": P.Options(pdhg_tolerance=1e-8, iteration_limit=1000000),
            "mixed": P.Options(pdhg_tolerance=1e-8, iteration_limit=1000000,
                               pdhg_precision="mixed", pdhg_algorithm="halpern"),
            "halpern": P.Options(pdhg_tolerance=1e-8, iteration_limit=1000000,
                                 pdhg_algorithm="halpern")}
    sols = {}
    batch = [(k, lp) for k, (_, lp, how) in enumerate(cs) if how == "batch"]
    for k, s in zip([k for k, _ in batch],
                    P.batch_solve([lp for _, lp in batch],
                                  P.Options(pdhg_tolerance=1e-6, iteration_limit=1000000,
                                            pdhg_algorithm="halpern"))):
        sols[k] = s
    for k, (_, lp, how) in enumerate(cs):
        if how != "batch":
            sols[k] = P.solve_pdhg(lp, opts[how])
    return [sols[k] for k in range(len(cs))]


def _gz(src, dst):
    with open(src, "rb") as f, gzip.GzipFile(dst, "wb", mtime=0) as g:
        shutil.copyfileobj(f, g)


def main():
    import sol_io

    out_dir = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "gpu_answers")
    os.makedirs(out_dir, exist_ok=True)
    cs = cases()
    sols = solve_all(cs)
    tmp = tempfile.mkdtemp()
    for (name, lp, _), s in zip(cs, sols):
        lp.name = name
        sol_io.write_mps(lp, os.path.join(tmp, name + ".mps"))
        sol_io.write_sol(lp, s, os.path.join(tmp, name + ".sol"))
        _gz(os.path.join(tmp, name + ".mps"), os.path.join(out_dir, name + ".mps.gz"))
        _gz(os.path.join(tmp, name + ".sol"), os.path.join(out_dir, name + ".sol.gz"))
        print(f"{name}: {s.status} {s.objective:.12g} ({s.iterations} iterations)")
    shutil.rmtree(tmp)


if __name__ == "__main__":
    main()
