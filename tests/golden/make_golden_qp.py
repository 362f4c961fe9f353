"""Generates tests/golden/reference_qp.json from the REFERENCE solver's own convex-QP engine
(qp::solve_convex_qp, src/qp/qp_condat_vu.cpp, compiled in place into oracle/_ref by
`make -C oracle ref`). For every case of QP_CASES it records what the reference returned:
status, iteration count, objective and a few invariants of the point. The CUDA QP path is
tested against it on machines without the reference tree.

    python tests/golden/make_golden_qp.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from sih26_b200 import lpgen  # noqa: E402

# (m, n, nonzeros per column, seed, maximize, tolerance, iteration limit)
QP_CASES = [
    (20, 50, 3, 11, False, 1e-6, 100000),
    (40, 100, 3, 3, False, 1e-8, 200000),
    (40, 100, 3, 12, True, 1e-6, 100000),
    (80, 200, 4, 13, False, 1e-6, 100000),
    (60, 150, 3, 14, False, 1e-12, 500),
]


def qp_case(spec):
    m, n, k, seed, maximize, _, _ = spec
    return lpgen.qp_planted(m, n, k, seed=seed, maximize=maximize)


def main():
    if not oracle.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    out = {"generator": "tests/golden/make_golden_qp.py", "cases": []}
    for spec in QP_CASES:
        lp = qp_case(spec)
        tol, limit = spec[5], spec[6]
        r = oracle.ref_qp_solve(lp, tolerance=tol, iteration_limit=limit)
        out["cases"].append({
            "spec": list(spec), "status": r.status, "iterations": r.iterations,
            "objective": r.objective, "dual_bound": r.dual_bound,
            "planted_objective": lp.optimal_objective,
            "x_sum": float(np.sum(r.col_value)), "row_dual_sum": float(np.sum(r.row_dual)),
        })
        print(spec, r.status, r.iterations, r.objective)
    path = os.path.join(HERE, "reference_qp.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out['cases'])} records to {path}")


if __name__ == "__main__":
    main()
