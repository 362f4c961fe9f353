"""Makes tests/golden/kkt_fuzz_120.npz: the 120 instances of the reference's cross-engine gate
(tests/unit/test_pdhg.cpp:178-222: oracle::kkt_lp from std::mt19937_64(20260904), at most 6
rows and 6 columns), drawn by the reference's own generator (oracle/_ref, ref_fuzz.cpp), with
each instance's analytic optimum and what the reference's solve_pdhg returns on it at
pdhg_tolerance 1e-9 (status, objective). Run here, where the reference tree exists:

    python tests/golden/make_kkt_fuzz.py

load() reads the fixture back on any machine.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SEED, MAX_ROWS, MAX_COLS, COUNT = 20260904, 6, 6, 120
KEYS = ("col_starts", "row_indices", "values", "cost", "col_lower", "col_upper", "row_lower",
        "row_upper")


def main():
    """Packs the instances into flat arrays: per instance its sizes, its analytic optimum and
    the reference's status and objective; the arrays concatenated in instance order."""
    import oracle

    flat = {k: [] for k in KEYS}
    meta, optimal, ref_obj, ref_status = [], [], [], []
    for k in range(COUNT):
        lp = oracle.ref_kkt_instance(SEED, MAX_ROWS, MAX_COLS, k)
        r = oracle.ref_solve(lp, tolerance=1e-9, iteration_limit=1000000)
        meta.append([lp.num_rows, lp.num_cols, lp.num_nonzeros, int(lp.maximize)])
        for key in KEYS:
            flat[key].append(np.asarray(getattr(lp, key)))
        optimal.append(lp.optimal_objective)
        ref_obj.append(r.objective)
        ref_status.append(r.status)
    out = {key: np.concatenate(v) for key, v in flat.items()}
    out.update(meta=np.array(meta, dtype=np.int64), optimal_objective=np.array(optimal),
               ref_objective=np.array(ref_obj), ref_status=np.array(ref_status))
    np.savez_compressed(os.path.join(HERE, "kkt_fuzz_120.npz"), **out)
    print(f"{COUNT} instances; the reference's solve_pdhg is optimal on "
          f"{sum(s == 'optimal' for s in ref_status)}")


def load():
    """The fixture's instances as lpgen.LP objects (optimal_objective = the analytic optimum),
    each with the reference's (status, objective)."""
    from sih26_b200.lpgen import LP

    d = np.load(os.path.join(HERE, "kkt_fuzz_120.npz"))
    at = {k: 0 for k in KEYS}
    out = []
    for k, (m, n, nnz, mx) in enumerate(d["meta"]):
        size = {"col_starts": n + 1, "row_indices": nnz, "values": nnz, "cost": n,
                "col_lower": n, "col_upper": n, "row_lower": m, "row_upper": m}
        arr = {}
        for key, length in size.items():
            arr[key] = d[key][at[key]:at[key] + length]
            at[key] += length
        lp = LP(num_rows=int(m), num_cols=int(n), maximize=bool(mx), name=f"kkt{k}",
                optimal_objective=float(d["optimal_objective"][k]), **arr)
        out.append((lp, str(d["ref_status"][k]), float(d["ref_objective"][k])))
    return out


if __name__ == "__main__":
    main()
