"""Convex QP on the GPU (sankhya_qp_gpu_solve) against the reference's own QP engine
(qp::solve_convex_qp, src/qp/qp_condat_vu.cpp): the golden fixture made by the reference build,
the planted optimum, the termination measures, and the convexity refusal."""
import json
import math
import os

import numpy as np
import pytest

from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_qp.json")


def _opts(**kw):
    o = P.Options()
    for k, v in kw.items():
        o.set(k, v)
    return o


@pytest.mark.parametrize("rec", json.load(open(GOLDEN))["cases"], ids=lambda r: str(r["spec"][:5]))
def test_matches_the_reference_qp_engine(rec):
    m, n, k, seed, maximize, tol, limit = rec["spec"]
    lp = lpgen.qp_planted(m, n, k, seed=seed, maximize=maximize)
    s = P.solve_qp(lp, _opts(qp_tolerance=tol, iteration_limit=limit))
    assert s.status == rec["status"], (s.status, s.message)
    # same steps, same algorithm; only the summation order differs, so the run ends at the
    # same termination check or one of its neighbours
    assert abs(s.iterations - rec["iterations"]) <= max(100, 0.05 * rec["iterations"]), (
        s.iterations, rec["iterations"])
    if rec["status"] == "optimal":
        assert abs(s.objective - rec["objective"]) <= 1e-6 * max(1.0, abs(rec["objective"]))
        assert abs(s.objective - rec["planted_objective"]) <= 1e-5 * abs(rec["planted_objective"])
        assert s.residuals["absolute_primal"] <= tol and s.residuals["absolute_dual"] <= tol
        assert s.dual_bound == s.objective
    else:
        assert s.iterations == limit and math.isinf(s.dual_bound)


def test_an_lp_through_the_qp_engine():
    lp = lpgen.uniform_planted(60, 150, 4, seed=2)
    s = P.solve_qp(lp, _opts(qp_tolerance=1e-7, iteration_limit=400000))
    assert s.status == "optimal", s.message
    assert abs(s.objective - lp.optimal_objective) <= 1e-5 * abs(lp.optimal_objective)


def test_non_convex_is_refused_like_the_reference():
    lp = lpgen.qp_planted(20, 50, 3, seed=5)
    lp.hessian_values = lp.hessian_values.copy()
    diag = [lp.hessian_col_starts[j] for j in range(5)]  # the first entry of a column is its diagonal
    lp.hessian_values[diag] = -1.0
    s = P.solve_qp(lp, _opts())
    assert s.status == "model_error" and "not convex" in s.message


def test_beyond_the_dense_test_needs_an_explicit_assumption():
    lp = lpgen.qp_planted(900, 2100, 3, seed=6)
    s = P.solve_qp(lp, _opts(qp_tolerance=1e-5, iteration_limit=20000))
    assert s.status == "model_error" and "could not be established" in s.message
    s = P.solve_qp(lp, _opts(qp_tolerance=1e-5, iteration_limit=200000, qp_assume_convex=True))
    assert s.status == "optimal", s.message
    assert abs(s.objective - lp.optimal_objective) <= 1e-4 * abs(lp.optimal_objective)
