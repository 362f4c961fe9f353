"""Shared LP cases for the parity tests.

The hand-written LPs restate the reference's own PDHG unit tests (tests/unit/test_pdhg.cpp),
each with the optimum its comment derives; the generated ones are seeded planted-optimum
instances from sih26_b200.lpgen.
"""
from __future__ import annotations

import math

from sih26_b200 import lpgen

INF = math.inf


def hand_cases():
    """(name, LP, expected objective or None, solve options) from test_pdhg.cpp."""
    out = []
    # test_pdhg.cpp:95-101  min x + y  s.t. x + y >= 2          -> 2
    out.append(("minimises_a_sum", lpgen.from_dense([[1, 1]], [2], [INF], [1, 1]), 2.0))
    # :103-109  min x + 2y  s.t. x + y = 4                     -> 4
    out.append(("equality_row", lpgen.from_dense([[1, 1]], [4], [4], [1, 2]), 4.0))
    # :111-118  2 <= x <= 6 as a range row, min x              -> 2
    out.append(("range_row", lpgen.from_dense([[1]], [2], [6], [1]), 2.0))
    # :120-126  min -x, x <= 100 by a row, x <= 7 by a bound    -> -7
    out.append(("column_upper_bound",
                lpgen.from_dense([[1]], [-INF], [100], [-1], col_upper=[7.0]), -7.0))
    # :128-138  max 3x + 5y, x <= 4, 2y <= 12, 3x + 2y <= 18    -> 36 at (2, 6)
    out.append(("original_sense",
                lpgen.from_dense([[1, 0], [0, 2], [3, 2]], [-INF] * 3, [4, 12, 18], [3, 5],
                                 maximize=True), 36.0))
    # :140-146  min x, x >= 3, offset 10                          -> 13
    out.append(("objective_offset",
                lpgen.from_dense([[1]], [3], [INF], [1], objective_offset=10.0), 13.0))
    # :224-242  min x + y, x + y >= 1e5 (relative and absolute measures diverge)
    out.append(("large_rhs", lpgen.from_dense([[1, 1]], [1e5], [INF], [1, 1]), 1e5))
    # :314-338  the blending model of demo/crude_blend.mps, built in memory
    blend = lpgen.from_dense([[1.0, 1.0, 1.0], [0.30, 0.45, 0.38], [0.80, -0.86, -0.22]],
                             [90.0, 40.0, -INF], [120.0, 40.0, 0.0], [2.40, 1.60, 1.64],
                             col_lower=[10.0, 0.0, 0.0], col_upper=[INF, 45.0, 60.0],
                             maximize=True, name="BLENDGUARD")
    out.append(("blend", blend, None))
    return out


def generated_cases():
    """Small seeded planted instances (name, LP)."""
    out = []
    for seed in (1, 2, 3):
        out.append((f"uniform_60x150_s{seed}", lpgen.uniform_planted(60, 150, 4, seed=seed)))
    out.append(("uniform_200x500_s7", lpgen.uniform_planted(200, 500, 5, seed=7)))
    return out


def netlib_cases():
    """The Netlib LPs of the reference tree (data/netlib/*.mps) as read by the reference's MPS
    reader, from tests/golden/netlib.npz (made by tests/golden/make_netlib.py): (LP, published
    optimum, the reference solve_pdhg's status and objective at pdhg_tolerance 1e-8)."""
    import os

    import numpy as np

    from sih26_b200.lpgen import LP

    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "netlib.npz"))
    names = sorted({k.split("/")[0] for k in d.files},
                   key=lambda nm: int(d[nm + "/meta"][0]) * int(d[nm + "/meta"][1]))
    out = []
    for nm in names:
        m, n, mx = (int(v) for v in d[nm + "/meta"])
        lp = LP(num_rows=m, num_cols=n, col_starts=d[nm + "/col_starts"],
                row_indices=d[nm + "/row_indices"], values=d[nm + "/values"],
                cost=d[nm + "/cost"], col_lower=d[nm + "/col_lower"],
                col_upper=d[nm + "/col_upper"], row_lower=d[nm + "/row_lower"],
                row_upper=d[nm + "/row_upper"], maximize=bool(mx),
                objective_offset=float(d[nm + "/objective_offset"]), name=nm)
        out.append((lp, float(d[nm + "/published_optimal"]), str(d[nm + "/ref_status"]),
                    float(d[nm + "/ref_objective"])))
    return out


def kkt_fuzz_cases():
    """The 120 instances of the reference's cross-engine gate (tests/unit/test_pdhg.cpp:178-222)
    from tests/golden/kkt_fuzz_120.npz: (LP with its analytic optimum, the reference
    solve_pdhg's status and objective at pdhg_tolerance 1e-9)."""
    import os
    import sys

    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    if here not in sys.path:
        sys.path.insert(0, here)
    import make_kkt_fuzz

    return make_kkt_fuzz.load()
