"""Makes tests/golden/netlib.npz: the Netlib LPs of the reference tree (data/netlib/*.mps),
read by the reference's own MPS reader (oracle/_ref, src/io/mps_reader.cpp), with the
published optima of data/netlib/reference.json and what the reference's solve_pdhg returns on
each (pdhg_tolerance 1e-8, restarts on, 1,000,000 iterations at most), so GPU tests can run
on boxes without the reference tree. Run here, where the tree and oracle/_ref exist:

    python tests/golden/make_netlib.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

REF = "/root/reference/data/netlib"
NAMES = ("afiro", "sc50a", "sc50b", "blend", "adlittle", "share2b", "sc105", "stocfor1",
         "israel")


def main():
    published = json.load(open(os.path.join(REF, "reference.json")))["instances"]
    out = {}
    for name in NAMES:
        lp = oracle.ref_read_model(os.path.join(REF, name + ".mps"))
        r = oracle.ref_solve(lp, tolerance=1e-8, iteration_limit=1000000)
        p = f"{name}/"
        out.update({p + "col_starts": lp.col_starts, p + "row_indices": lp.row_indices,
                    p + "values": lp.values, p + "cost": lp.cost, p + "col_lower": lp.col_lower,
                    p + "col_upper": lp.col_upper, p + "row_lower": lp.row_lower,
                    p + "row_upper": lp.row_upper,
                    p + "meta": np.array([lp.num_rows, lp.num_cols, int(lp.maximize)]),
                    p + "objective_offset": np.array(lp.objective_offset),
                    p + "published_optimal": np.array(published[name]["published_optimal"]),
                    p + "ref_objective": np.array(r.objective),
                    p + "ref_iterations": np.array(r.iterations),
                    p + "ref_status": np.array(r.status)})
        print(f"{name}: {lp.num_rows} x {lp.num_cols}, {lp.num_nonzeros} nonzeros; reference "
              f"{r.status} in {r.iterations} iterations, objective {r.objective:.10g} "
              f"(published {published[name]['published_optimal']})")
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "netlib.npz"),
                        **out)


if __name__ == "__main__":
    main()
