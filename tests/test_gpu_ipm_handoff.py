"""The GPU answer handed to the reference's interior-point polish.

When PDHG stops short of the project's standard, the reference polishes its answer with the
interior point warm-started from (col_value, row_dual, col_dual), and the merged answer reads
"pdhg-cpu+ipm" (polish_with_the_interior_point, src/core/solve.cpp:184-243; ipm::WarmStart,
include/sankhya/ipm.hpp:24-34). The GPU engine drops in before that step, so its answer must
be a warm start the reference's interior point accepts: here the GPU stops early (an
iteration limit, or the relative-KKT rule at a loose tolerance), the reference's polish
(oracle/_ref: the reference's src/ipm/ipm.cpp in the polish's own steps) takes over, and the
result must be optimal at the LP's optimum (the planted one; for the maximised LP the
reference solver's own) with the algorithm "pdhg-gpu+ipm".
"""
import pytest

import oracle
from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(),
                                 reason="reference build (oracle/_ref) not present")]


def _lps():
    big = lpgen.uniform_planted(300, 750, 6, seed=9)
    big.maximize = True
    return [("uniform", lpgen.uniform_planted(2000, 5000, 10, seed=0)), ("uniform_max", big),
            ("block_angular", lpgen.block_angular_planted(blocks=4, block_rows=60,
                                                          block_cols=150, nnz_per_col=4,
                                                          linking_rows=8, seed=4))]


STOPS = {"iteration_limit": dict(iteration_limit=400),
         "loose_relative_kkt": dict(pdhg_tolerance=1e-3, pdhg_stop_rule="relative_kkt")}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("stop", sorted(STOPS))
@pytest.mark.parametrize("name,lp", _lps(), ids=[n for n, _ in _lps()])
def test_gpu_answer_polished_by_the_reference_interior_point(name, lp, stop, precision):
    opts = P.Options(pdhg_precision=precision, pdhg_algorithm="halpern", **STOPS[stop])
    s = P.solve_pdhg(lp, opts)
    if s.status == "optimal":
        pytest.skip("this stop already met the standard; nothing to polish")
    assert s.status in ("feasible", "iteration_limit"), (name, s.status)
    q = s.quality
    worst = max(q["primal_infeasibility_scaled"], q["dual_infeasibility_scaled"])
    p = oracle.ref_polish_ipm(lp, s.col_value, s.row_dual, s.col_dual, s.status, s.iterations,
                              s.algorithm, worst)
    assert p["polished"], (name, p["message"])
    assert p["status"] == "optimal", (name, p["status"], p["message"])
    assert p["algorithm"] == "pdhg-gpu+ipm"
    assert p["iterations"] == s.iterations + p["polish_iterations"]
    # the optimum: the planted one, or for the maximised LP (whose planted point was built for
    # the minimise sense) what the reference's own solve_pdhg reaches at 1e-9
    want = (lp.optimal_objective if not lp.maximize
            else oracle.ref_solve(lp, tolerance=1e-9, iteration_limit=1000000).objective)
    assert abs(p["objective"] - want) <= 1e-6 * max(1.0, abs(want)), (name, p["objective"], want)
