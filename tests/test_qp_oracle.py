"""The QP oracle: the reference's own convex-QP engine (src/qp/qp_condat_vu.cpp, through the
reference build) on the planted QP family, and the golden fixture the GPU tests use."""
import json
import os

import numpy as np
import pytest

import oracle
from sih26_b200 import lpgen

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_qp.json")
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="needs the reference build")


def test_planted_qp_is_convex_and_its_optimum_satisfies_kkt():
    lp = lpgen.qp_planted(30, 80, 3, seed=1)
    n = lp.num_cols
    q = np.zeros((n, n))
    for j in range(n):
        for k in range(lp.hessian_col_starts[j], lp.hessian_col_starts[j + 1]):
            i = lp.hessian_row_indices[k]
            q[i, j] = q[j, i] = lp.hessian_values[k]
    assert np.linalg.eigvalsh(q).min() > 0.0
    a = lp.to_scipy_csc()
    x = lp.x_star
    assert np.allclose(a @ x, lp.row_lower)
    # stationarity with complementary reduced costs: c + Qx* - A'lam = z
    z = lp.cost + q @ x - a.T @ lp.row_dual_star
    assert np.all(z[x <= 1e-12] >= 0.1 - 1e-9)
    assert np.all(z[x >= lp.col_upper - 1e-12] <= -0.1 + 1e-9)
    interior = (x > 1e-12) & (x < lp.col_upper - 1e-12)
    assert np.allclose(z[interior], 0.0, atol=1e-9)


@needs_ref
def test_golden_fixture_is_what_the_reference_returns():
    golden = json.load(open(GOLDEN))
    for rec in golden["cases"]:
        m, n, k, seed, maximize, tol, limit = rec["spec"]
        lp = lpgen.qp_planted(m, n, k, seed=seed, maximize=maximize)
        r = oracle.ref_qp_solve(lp, tolerance=tol, iteration_limit=limit)
        assert (r.status, r.iterations) == (rec["status"], rec["iterations"])
        assert r.objective == rec["objective"]


@needs_ref
def test_reference_reaches_the_planted_optimum():
    for spec in json.load(open(GOLDEN))["cases"]:
        if spec["status"] != "optimal":
            continue
        assert abs(spec["objective"] - spec["planted_objective"]) <= 1e-5 * abs(spec["planted_objective"])
