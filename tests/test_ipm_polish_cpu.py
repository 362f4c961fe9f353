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
