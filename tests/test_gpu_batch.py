"""The batched / served engine: many uneven LPs per launch, per-LP termination, Farkas
certificates for the infeasible ones, and the same answer alone and in the mix."""
import numpy as np
import pytest

import oracle
from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _opts(**kw):
    o = P.Options(pdhg_tolerance=TOL, pdhg_stop_rule="relative_kkt", iteration_limit=200000)
    for k, v in kw.items():
        o.set(k, v)
    return o


def _farkas_ok(lp, y):
    """src/core/certificate.cpp:29-119, through the reference build when it is present."""
    if oracle.ref_available():
        ok, why = oracle.ref_farkas_check(lp, y)
        return ok, why
    fin = lambda v: np.abs(v) < 1e30  # noqa: E731
    if not np.any(y != 0):
        return False, "zero"
    if np.any((y > 0) & ~fin(lp.row_lower)) or np.any((y < 0) & ~fin(lp.row_upper)):
        return False, "missing row bound"
    required = float(np.sum(np.where(y > 0, y * np.where(fin(lp.row_lower), lp.row_lower, 0),
                                      y * np.where(fin(lp.row_upper), lp.row_upper, 0))))
    a = lp.to_scipy_csc()
    d = a.T @ y
    scale = float(abs(a.multiply(y[:, None])).max()) if lp.num_nonzeros else 0.0
    thr = 1e-11 * max(1.0, scale)
    reach = float(np.sum(np.where(d > thr, d * lp.col_upper, 0.0) + np.where(d < -thr, d * lp.col_lower, 0.0)))
    margin = required - reach
    return margin > 1e-7 * max(1.0, abs(required), abs(reach), scale), f"margin {margin}"


@pytest.fixture(scope="module")
def batch():
    lps = lpgen.uneven_batch(count=48, m_lo=50, m_hi=600, infeasible_fraction=0.2, seed=11)
    sols = P.batch_solve(lps, _opts())
    return lps, sols


def test_every_feasible_lp_meets_the_tolerance(batch):
    lps, sols = batch
    checked = 0
    for lp, s in zip(lps, sols):
        if lp.farkas_star is not None:
            continue
        assert s.status in ("optimal", "feasible"), (lp.name, s.status, s.message)
        # the bar is the request itself: relative KKT <= 1e-6 recomputed from the point
        r = oracle.oracle_evaluate(lp, s.col_value, -s.row_dual)
        assert max(r["primal"], r["dual"], r["gap"]) <= TOL, (lp.name, r)
        # and the planted optimum to the accuracy such a point carries
        scale = max(1.0, abs(lp.optimal_objective))
        assert abs(s.objective - lp.optimal_objective) <= 1e-4 * scale, lp.name
        checked += 1
    assert checked >= 30


def test_infeasible_lps_come_back_with_a_checked_certificate(batch):
    lps, sols = batch
    n_inf = 0
    for lp, s in zip(lps, sols):
        if lp.farkas_star is None:
            continue
        n_inf += 1
        assert s.status == "infeasible", (lp.name, s.status, s.message)
        ok, why = _farkas_ok(lp, s.farkas_dual)
        assert ok, (lp.name, why)
    assert n_inf >= 5


def test_same_answer_alone_and_in_the_mix(batch):
    lps, sols = batch
    for k in (0, 7, 19):
        alone = P.batch_solve([lps[k]], _opts())[0]
        assert alone.status == sols[k].status
        assert alone.iterations == sols[k].iterations
        assert np.array_equal(alone.col_value, sols[k].col_value)
        assert np.array_equal(alone.row_dual, sols[k].row_dual)


def test_batch_agrees_with_the_single_lp_path(batch):
    lps, sols = batch
    for k in range(6):
        if lps[k].farkas_star is not None:
            continue
        single = P.solve_pdhg(lps[k], _opts())
        assert single.status == sols[k].status
        # both points have relative gap <= TOL, so each objective is within
        # TOL * (1 + |p| + |d|) of the optimum: the two differ by at most twice that
        bound = 2 * TOL * (1.0 + 2 * abs(single.objective))
        assert abs(single.objective - sols[k].objective) <= bound


def test_server_admits_while_others_run_and_matches_the_batch(batch):
    lps, sols = batch
    with P.Server(chunk_attempts=256) as srv:
        first = [srv.submit(lp, _opts()) for lp in lps[:20]]
        srv.step()
        srv.step()
        later = [srv.submit(lp, _opts()) for lp in lps[20:]]
        results = {}
        for _ in range(100000):
            active, waiting, _ = srv.step()
            for t in list(srv.pending):
                r = srv.result(t)
                if r is not None:
                    results[t] = r
            if active == 0 and waiting == 0 and not srv.pending:
                break
    tickets = first + later
    for k, t in enumerate(tickets):
        r = results[t]
        assert r.status == sols[k].status
        assert r.iterations == sols[k].iterations  # chunking pauses, it changes nothing
        assert np.array_equal(r.col_value, sols[k].col_value)


def test_cluster_class_meets_the_tolerance_and_is_the_same_alone(batch):
    """Every LP forced onto 8-block clusters: same bar, and the same bits alone and in the mix."""
    lps, sols = batch
    subset = lps[:16]
    with P.Server(chunk_attempts=0, cluster_min_nnz=1, clusters=4) as srv:
        got = srv.solve_all(subset, _opts())
    for lp, s, ref in zip(subset, got, sols):
        assert s.status == ref.status, (lp.name, s.status, ref.status)
        if lp.farkas_star is not None:
            ok, why = _farkas_ok(lp, s.farkas_dual)
            assert ok, (lp.name, why)
            continue
        r = oracle.oracle_evaluate(lp, s.col_value, -s.row_dual)
        assert max(r["primal"], r["dual"], r["gap"]) <= TOL, (lp.name, r)
    with P.Server(chunk_attempts=0, cluster_min_nnz=1, clusters=4) as srv:
        alone = srv.solve_all([subset[3]], _opts())[0]
    assert alone.iterations == got[3].iterations
    assert np.array_equal(alone.col_value, got[3].col_value)


def test_both_classes_in_one_server_match_their_own_runs(batch):
    """A threshold that splits the batch: each LP gets what its class gives it alone."""
    lps, sols = batch
    nnz = sorted(lp.num_nonzeros for lp in lps)
    cut = nnz[len(nnz) // 2]
    with P.Server(chunk_attempts=512, cluster_min_nnz=cut, clusters=4) as srv:
        mixed = srv.solve_all(lps, _opts())
    big = [k for k, lp in enumerate(lps) if lp.num_nonzeros >= cut]
    small = [k for k in range(len(lps)) if lps[k].num_nonzeros < cut]
    assert big and small
    for k in small[:6]:
        assert mixed[k].iterations == sols[k].iterations
        assert np.array_equal(mixed[k].col_value, sols[k].col_value)
    with P.Server(chunk_attempts=0, cluster_min_nnz=1, clusters=4) as srv:
        own = srv.solve_all([lps[k] for k in big[:6]], _opts())
    for k, o in zip(big[:6], own):
        assert mixed[k].status == o.status
        assert mixed[k].iterations == o.iterations
        assert np.array_equal(mixed[k].col_value, o.col_value)
