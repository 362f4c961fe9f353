"""Generates tests/golden/reference_pdhg.json from the REFERENCE solver's own PDHG.

Run here, where the reference tree exists and `make -C oracle ref` has built
oracle/_ref/libsankhya_ref.so (the reference's src/pdhg, src/la, src/core sources compiled in
place with our harness). The fixture records, for every case in tests/cases.py and every
option set below, what sankhya::pdhg::solve_pdhg returned: status, iteration count,
objective, dual bound and a few invariants of the point. The oracle restatement and the
CUDA path are tested against it on machines without the reference tree.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import oracle  # noqa: E402
from cases import generated_cases, hand_cases  # noqa: E402

OPTION_SETS = [
    dict(tolerance=1e-8, iteration_limit=200000, restart=True, stop_at_request=False),
    dict(tolerance=1e-4, iteration_limit=200000, restart=True, stop_at_request=True),
    dict(tolerance=1e-6, iteration_limit=200000, restart=False, stop_at_request=False),
    dict(tolerance=1e-12, iteration_limit=20, restart=True, stop_at_request=False),
]


def main():
    if not oracle.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    out = {"generator": "tests/golden/make_golden.py", "cases": []}
    cases = [(n, lp) for n, lp, _ in hand_cases()] + generated_cases()
    for name, lp in cases:
        for k, opts in enumerate(OPTION_SETS):
            r = oracle.ref_solve(lp, **opts)
            out["cases"].append({
                "case": name, "options": k, **{f"opt_{a}": b for a, b in opts.items()},
                "status": r.status, "iterations": r.iterations,
                "objective": r.objective, "dual_bound": r.dual_bound,
                "x_sum": float(np.sum(r.col_value)),
                "row_dual_sum": float(np.sum(r.row_dual)),
                "col_value": r.col_value.tolist() if lp.num_cols <= 8 else None,
            })
    path = os.path.join(HERE, "reference_pdhg.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print(f"wrote {len(out['cases'])} records to {path}")


if __name__ == "__main__":
    main()
