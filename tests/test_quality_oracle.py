"""The numpy restatement of Solution::recompute_quality (oracle/quality.py) against the
reference's own recompute_quality (src/core/model.cpp:228-424) compiled from its sources.

Points: the reference solver's own answers on the hand-written and generated LPs, and the
same answers disturbed so that every measure has something to find (bound and row
violations, wrong-signed prices and reduced costs, col_dual out of step with c - A'y, slack
with a price on it). Equality is bit for bit.
"""
import math

import numpy as np
import pytest

import oracle
from sih26_b200 import lpgen
from tests.cases import generated_cases, hand_cases

needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference build (oracle/_ref) not present")


def edge_lps():
    """Every bound kind at once: a free column, a fixed one, a boxed one; >=, <=, range and
    equality rows; both senses, with an objective offset."""
    inf = math.inf
    rows = [[1, 1, 1, 0], [1, 0, -1, 0], [0, 1, 1, 0], [0, 1, 0, -1]]
    kw = dict(col_lower=[0, -inf, 1, -inf], col_upper=[5, inf, 1, inf])
    return [("edge_min", lpgen.from_dense(rows, [1, -inf, 0, 0], [inf, 2, 3, 0], [1, 2, -1, 0],
                                          name="edge_min", **kw)),
            ("edge_max", lpgen.from_dense(rows, [1, -inf, 0, 0], [inf, 2, 3, 0], [-1, -2, 1, 0],
                                          maximize=True, objective_offset=3.5, name="edge_max",
                                          **kw))]


def _lps():
    out = [(name, lp) for name, lp, _ in hand_cases()]
    out += edge_lps()
    out += generated_cases()
    out.append(("block_angular", lpgen.block_angular_planted(blocks=3, block_rows=40,
                                                             block_cols=100, nnz_per_col=4,
                                                             linking_rows=6, seed=4)))
    big = lpgen.uniform_planted(60, 150, 4, seed=9)
    big.maximize = True
    out.append(("uniform_max", big))
    return out


def _same(a, b):
    for k in a:
        va, vb = a[k], b[k]
        assert (va == vb) or (math.isnan(va) and math.isnan(vb)), (k, va, vb)


@needs_ref
@pytest.mark.parametrize("name,lp", _lps(), ids=[n for n, _ in _lps()])
def test_restatement_matches_reference(name, lp):
    r = oracle.ref_solve(lp, tolerance=1e-8, iteration_limit=20000)
    pts = [(r.col_value, r.row_dual, r.col_dual, r.dual_bound)]
    rng = np.random.default_rng(len(name))
    for scale in (1e-6, 1e-2, 1.0):
        x = r.col_value + scale * rng.standard_normal(lp.num_cols)
        rd = r.row_dual + scale * rng.standard_normal(lp.num_rows)
        cd = r.col_dual + scale * rng.standard_normal(lp.num_cols)
        pts.append((x, rd, cd, r.objective - scale))
    for x, rd, cd, bound in pts:
        got = oracle.recompute_quality(lp, x, rd, cd, bound)
        want = oracle.ref_recompute_quality(lp, x, rd, cd, bound)
        _same(got, want)


@needs_ref
def test_disturbed_points_find_every_measure():
    lp = lpgen.uniform_planted(60, 150, 4, seed=1)
    r = oracle.ref_solve(lp, tolerance=1e-8, iteration_limit=20000)
    rng = np.random.default_rng(3)
    x = r.col_value + 0.1 * rng.standard_normal(lp.num_cols)
    cd = r.col_dual + 0.1 * rng.standard_normal(lp.num_cols)
    q = oracle.recompute_quality(lp, x, r.row_dual, cd, r.dual_bound)
    for k in ("primal_infeasibility", "primal_infeasibility_scaled", "dual_infeasibility",
              "dual_infeasibility_scaled", "complementarity_violation"):
        assert q[k] > 1e-3, (k, q[k])
    _same(q, oracle.ref_recompute_quality(lp, x, r.row_dual, cd, r.dual_bound))
