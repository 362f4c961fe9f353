"""The quality block of every answer (Solution::recompute_quality, src/core/model.cpp:228-424),
measured on the device, against the numpy restatement (oracle/quality.py, pinned bit for bit
to the reference's recompute_quality by tests/test_quality_oracle.py) on the same reported
point.

Single-LP solves (both operators, both precisions), the batched engine and the resident
server; converged points, where every measure is a rounding residue, and points stopped
early, where every measure has something to find. The device forms the row and column sums
in another order and each matrix term from the scaled values, so each figure may differ by
rounding: at most 1e-9 of its value plus 1e-12 of the largest term it was measured from.
"""
import math

import numpy as np
import pytest

import oracle
from sih26_b200 import lpgen
from sih26_b200 import pdhg as P
from tests.cases import generated_cases, hand_cases
from tests.test_quality_oracle import edge_lps

pytestmark = pytest.mark.gpu

KEYS = ("primal_infeasibility", "primal_infeasibility_scaled", "dual_infeasibility",
        "dual_infeasibility_scaled", "complementarity_violation", "absolute_gap",
        "relative_gap")


def _term_scale(lp, s):
    a = float(np.max(np.abs(lp.values))) if lp.num_nonzeros else 1.0
    v = [1.0, float(np.max(np.abs(lp.cost)))]
    for arr in (s.col_value, s.row_dual, s.col_dual):
        if arr is not None and arr.size:
            v.append(float(np.max(np.abs(arr))))
    return max(v) * max(1.0, a)


def _check(lp, s):
    assert s.quality is not None, s.status
    want = oracle.recompute_quality(lp, s.col_value, s.row_dual, s.col_dual, s.dual_bound)
    assert s.objective == want["objective"]
    term = _term_scale(lp, s)
    for k in KEYS:
        g, w = s.quality[k], want[k]
        if math.isinf(w) or math.isinf(g):
            assert g == w, (lp.name, k, g, w)
            continue
        assert abs(g - w) <= 1e-9 * abs(w) + 1e-12 * term, (lp.name, k, g, w)
    assert s.quality["primal_infeasibility"] == s.primal_infeasibility


def _lps():
    out = [lp for _, lp, _ in hand_cases()] + [lp for _, lp in generated_cases()]
    out += [lp for _, lp in edge_lps()]
    out.append(lpgen.block_angular_planted(blocks=3, block_rows=40, block_cols=100,
                                           nnz_per_col=4, linking_rows=6, seed=4))
    mx = lpgen.uniform_planted(60, 150, 4, seed=9)
    mx.maximize = True
    out.append(mx)
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("algorithm", ["reference", "halpern"])
def test_single_lp_quality_matches_the_restatement(precision, algorithm):
    for lp in _lps():
        for limit in (200000, 150):
            s = P.solve_pdhg(lp, P.Options(pdhg_tolerance=1e-8, iteration_limit=limit,
                                           pdhg_precision=precision,
                                           pdhg_algorithm=algorithm))
            if s.status in ("infeasible", "unbounded", "model_error"):
                continue
            _check(lp, s)


def test_early_stop_has_something_to_measure():
    lp = lpgen.uniform_planted(200, 500, 5, seed=7)
    s = P.solve_pdhg(lp, P.Options(pdhg_tolerance=1e-10, iteration_limit=120,
                                   pdhg_precision="fp64"))
    assert s.status == "iteration_limit"
    for k in ("primal_infeasibility", "dual_infeasibility_scaled", "complementarity_violation"):
        assert s.quality[k] > 1e-6, (k, s.quality[k])
    _check(lp, s)


def test_large_lp_quality_through_device_preparation():
    lp = lpgen.powerlaw_planted(20000, 50000, 10, seed=3)
    s = P.solve_pdhg(lp, P.Options(pdhg_tolerance=1e-6, pdhg_stop_rule="relative_kkt",
                                   pdhg_precision="mixed", pdhg_algorithm="halpern",
                                   iteration_limit=4000))
    _check(lp, s)


def test_batched_and_served_quality_matches_the_restatement():
    rng = np.random.default_rng(11)
    lps = [lpgen.small_planted(int(m), int(m * 2.5), 3, 8, rng) for m in (40, 90, 300, 1200)]
    lps += _lps()[-2:]
    opts = P.Options(pdhg_tolerance=1e-7, pdhg_stop_rule="relative_kkt", iteration_limit=200000)
    for lp, s in zip(lps, P.batch_solve(lps, opts)):
        if s.status in ("infeasible", "unbounded"):
            continue
        _check(lp, s)
    short = P.Options(pdhg_tolerance=1e-12, iteration_limit=100)
    with P.Server(chunk_attempts=64) as srv:
        for lp, s in zip(lps, srv.solve_all(lps, short)):
            _check(lp, s)
