"""Large LPs in the served engine go to the single-LP engine.

A resident server routes every LP with at least solo_min_nnz nonzeros to the single-LP
engine, one per step on the whole GPU between its batched launches (sankhya_pdhg_server_config
.solo_min_nnz): at that size one LP fills the GPU by itself. The answers of routed LPs must be
bit-for-bit those of sankhya_pdhg_gpu_solve with the same params, the others those of the
batched engine, and every answer must meet the request (checked by the oracle) or carry a
certificate the reference's checkers accept.
"""
import numpy as np
import pytest

import oracle
from certs import farkas_ok
from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = pytest.mark.gpu


def test_server_routes_large_lps_to_the_single_lp_engine():
    rng = np.random.default_rng(21)
    lps = [lpgen.uniform_planted(60 + 40 * k, 150 + 100 * k, 5, seed=70 + k) for k in range(10)]
    lps[3] = lpgen.make_infeasible(lps[3], rng)
    lps[8] = lpgen.make_infeasible(lps[8], rng)
    opts = P.Options(pdhg_tolerance=1e-6, iteration_limit=200000, pdhg_algorithm="halpern",
                     pdhg_stop_rule="relative_kkt")
    threshold = 2500
    with P.Server(solo_min_nnz=threshold) as srv:
        got = srv.solve_all(lps, opts)
    batched = P.batch_solve([lp for lp in lps if lp.num_nonzeros < threshold], opts)
    small = iter(batched)
    solo = 0
    for lp, s in zip(lps, got):
        want = P.solve_pdhg(lp, opts) if lp.num_nonzeros >= threshold else next(small)
        solo += lp.num_nonzeros >= threshold
        assert s.status == want.status and s.iterations == want.iterations, lp.name
        for f in ("col_value", "row_dual", "col_dual"):
            assert np.array_equal(getattr(s, f), getattr(want, f)), (lp.name, f)
        if lp.farkas_star is not None:
            assert s.status == "infeasible" and farkas_ok(lp, s.farkas_dual)[0], lp.name
        else:
            assert s.status in ("optimal", "feasible"), (lp.name, s.status)
            r = oracle.oracle_evaluate(lp, s.col_value, -s.row_dual)
            assert max(r["primal"], r["dual"], r["gap"]) <= 1e-6, (lp.name, r)
    assert 3 <= solo < len(lps)
