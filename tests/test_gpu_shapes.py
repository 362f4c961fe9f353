"""LP shapes beyond the small parity cases, on the GPU.

* The batched engine on the upper end of the batched family (m log-uniform on [2,000, 5,000],
  5-15 nonzeros per column, 10 % infeasible; every LP from 16,384 nonzeros on an 8-block
  cluster): every feasible LP meets relative KKT 1e-6 recomputed by the oracle from its point,
  every infeasible one carries a Farkas certificate the reference's checker accepts.
* The autotuner on a block-angular LP whose linking rows hold more than 512 nonzeros each
  (segments of long rows in both phases): the measured schedule is cached and reused with the
  same bits, and the answer meets the request.
"""
import numpy as np
import pytest

import oracle
from certs import farkas_ok
from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = pytest.mark.gpu


def test_batched_engine_on_the_upper_end_of_the_batched_family():
    lps = lpgen.uneven_batch(count=24, m_lo=2000, m_hi=5000, infeasible_fraction=0.1, seed=17)
    assert sum(lp.num_nonzeros >= 16384 for lp in lps) >= 20
    sols = P.batch_solve(lps, P.Options(pdhg_tolerance=1e-6, pdhg_stop_rule="relative_kkt",
                                        pdhg_algorithm="halpern", iteration_limit=400000))
    for lp, s in zip(lps, sols):
        if lp.farkas_star is not None:
            assert s.status == "infeasible", (lp.name, s.status, s.message)
            assert farkas_ok(lp, s.farkas_dual)[0], lp.name
            continue
        assert s.status in ("optimal", "feasible"), (lp.name, s.status, s.message)
        r = oracle.oracle_evaluate(lp, s.col_value, -s.row_dual)
        assert max(r["primal"], r["dual"], r["gap"]) <= 1e-6, (lp.name, r)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autotune_on_long_linking_rows(tmp_path, monkeypatch, precision):
    monkeypatch.setenv("SANKHYA_PDHG_AUTOTUNE_CACHE", str(tmp_path / "autotune.tsv"))
    lp = lpgen.block_angular_planted(blocks=8, block_rows=400, block_cols=1000, nnz_per_col=6,
                                     linking_rows=40, linking_density=0.1, seed=6)
    lens = np.diff(lp.to_scipy_csc().tocsr().indptr)
    assert lens.max() > 512  # the linking rows are long rows
    opts = P.Options(pdhg_tolerance=1e-6, pdhg_stop_rule="relative_kkt", pdhg_autotune=True,
                     pdhg_precision=precision, pdhg_algorithm="halpern", iteration_limit=400000)
    first = P.solve_pdhg(lp, opts)
    second = P.solve_pdhg(lp, opts)
    assert first.autotuned == 1 and second.autotuned == 2
    assert second.schedule == first.schedule and second.iterations == first.iterations
    assert np.array_equal(second.col_value, first.col_value)
    assert first.status in ("optimal", "feasible"), first.message
    r = oracle.oracle_evaluate(lp, first.col_value, -first.row_dual)
    assert max(r["primal"], r["dual"], r["gap"]) <= 1e-6, r
    assert abs(first.objective - lp.optimal_objective) <= 1e-4 * abs(lp.optimal_objective)
