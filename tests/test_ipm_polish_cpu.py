"""The reference's interior-point polish harness (oracle/_ref, ref_polish_ipm) on the CPU: the
reference's own PDHG answer stopped early is polished to the planted optimum and named
"pdhg-cpu+ipm", as src/core/solve.cpp:184-243 does. The GPU's answers go through the same
harness in tests/test_gpu_ipm_handoff.py."""
import pytest

import oracle
from sih26_b200 import lpgen

needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference build (oracle/_ref) not present")


@needs_ref
def test_reference_answer_stopped_early_is_polished():
    lp = lpgen.uniform_planted(300, 750, 6, seed=9)
    r = oracle.ref_solve(lp, tolerance=1e-8, iteration_limit=300)
    assert r.status == "iteration_limit"
    q = oracle.recompute_quality(lp, r.col_value, r.row_dual, r.col_dual, r.dual_bound)
    worst = max(q["primal_infeasibility_scaled"], q["dual_infeasibility_scaled"])
    p = oracle.ref_polish_ipm(lp, r.col_value, r.row_dual, r.col_dual, r.status, r.iterations,
                              "pdhg-cpu", worst)
    assert p["polished"] and p["status"] == "optimal", p["message"]
    assert p["algorithm"] == "pdhg-cpu+ipm"
    assert abs(p["objective"] - lp.optimal_objective) <= 1e-6 * abs(lp.optimal_objective)


@needs_ref
def test_polish_finishes_an_iteration_limited_point_to_the_known_answer():
    """tests/unit/test_pdhg.cpp:642-660: min -3x - 5y s.t. x <= 4, 2y <= 12, 3x + 2y <= 18,
    PDHG stopped at 20 iterations on purpose, then polished: optimal at -36, (2, 6), named
    "pdhg-cpu+ipm", the count the sum of both phases, the message saying so."""
    import math

    lp = lpgen.from_dense([[1.0, 0.0], [0.0, 2.0], [3.0, 2.0]], [-math.inf] * 3,
                          [4.0, 12.0, 18.0], [-3.0, -5.0])
    r = oracle.ref_solve(lp, tolerance=1e-4, iteration_limit=20)
    assert r.status == "iteration_limit" and r.iterations == 20
    q = oracle.recompute_quality(lp, r.col_value, r.row_dual, r.col_dual, r.dual_bound)
    worst = max(q["primal_infeasibility_scaled"], q["dual_infeasibility_scaled"])
    p = oracle.ref_polish_ipm(lp, r.col_value, r.row_dual, r.col_dual, r.status, r.iterations,
                              "pdhg-cpu", worst, message=r.message)
    assert p["status"] == "optimal", p["message"]
    assert p["algorithm"] == "pdhg-cpu+ipm"
    assert abs(p["objective"] + 36.0) <= 1e-6
    assert abs(p["col_value"][0] - 2.0) <= 1e-5 and abs(p["col_value"][1] - 6.0) <= 1e-5
    assert p["polish_iterations"] > 0
    assert p["iterations"] == 20 + p["polish_iterations"]
    assert p["primal_infeasibility"] <= 1e-7
    assert p["message"].startswith(r.message + "; polished by the interior point in "
                                   f"{p['polish_iterations']} iterations"), p["message"]
