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
