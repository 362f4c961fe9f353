"""The Halpern operator (pdhg_algorithm = halpern): reflected restarted Halpern PDHG with the
reference's candidates, restart rules, primal weight, stopping test and status rules. It
changes the iterate path, not the answer: the same parity bar as the reference operator --
the reference's unit-test answers, the oracle's objective and active-bound pattern, the
request met by residuals recomputed from the returned point, certificates that pass the
reference's checkers, bit-for-bit repeatability."""
import numpy as np
import pytest

import oracle
from cases import generated_cases, hand_cases
from certs import farkas_ok, ray_ok
from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = pytest.mark.gpu


def _opts(**kw):
    o = P.Options(pdhg_algorithm="halpern")
    for k, v in kw.items():
        o.set(k, v)
    return o


def _y_pdhg_sign(lp, sol):
    sense = -1.0 if lp.maximize else 1.0
    return -sense * sol.row_dual


def _pattern(lp, x, tol=1e-6):
    lo = np.where(np.abs(lp.col_lower) < 1e30, lp.col_lower, -np.inf)
    hi = np.where(np.abs(lp.col_upper) < 1e30, lp.col_upper, np.inf)
    at_lo = np.abs(x - lo) <= tol * np.maximum(1.0, np.abs(lo))
    at_hi = np.abs(x - hi) <= tol * np.maximum(1.0, np.abs(hi))
    return np.where(at_lo, -1, np.where(at_hi, 1, 0))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name,lp,expected", hand_cases())
def test_reference_unit_test_answers(name, lp, expected, precision):
    s = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-8, iteration_limit=200000,
                               pdhg_precision=precision))
    assert s.status == "optimal", (name, s.message)
    if expected is not None:
        assert abs(s.objective - expected) <= 1e-6 * max(1.0, abs(expected)), name
    if name == "original_sense":
        assert abs(s.col_value[0] - 2.0) < 1e-4 and abs(s.col_value[1] - 6.0) < 1e-4
    if name == "blend":
        assert abs(s.objective - 214.14594594594595) < 1e-4
    assert s.primal_infeasibility <= 1e-7


@pytest.mark.parametrize("name,lp", generated_cases())
def test_generated_against_oracle(name, lp):
    tol = 1e-8
    s = P.solve_pdhg(lp, _opts(pdhg_tolerance=tol))
    o = oracle.oracle_solve(lp, tolerance=tol)
    assert s.status == o.status == "optimal", s.message
    scale = max(1.0, abs(o.objective))
    assert abs(s.objective - o.objective) <= 1e-6 * scale
    r = oracle.oracle_evaluate(lp, s.col_value, _y_pdhg_sign(lp, s))
    assert max(r["primal"], r["dual"], r["gap"]) <= tol
    assert r["absolute_primal"] <= 1e-7 and r["gap_as_verified"] <= 1e-9
    assert np.array_equal(_pattern(lp, s.col_value), _pattern(lp, o.col_value))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_2000x5000_to_1e6_and_fewer_iterations(precision):
    lp = lpgen.uniform_planted(2000, 5000, 10, seed=0)
    tol = 1e-6
    h = P.solve_pdhg(lp, _opts(pdhg_tolerance=tol, pdhg_stop_rule="relative_kkt",
                               pdhg_precision=precision))
    r = P.solve_pdhg(lp, P.Options(pdhg_tolerance=tol, pdhg_stop_rule="relative_kkt",
                                   pdhg_precision=precision))
    assert h.status in ("optimal", "feasible"), h.message
    res = oracle.oracle_evaluate(lp, h.col_value, _y_pdhg_sign(lp, h))
    assert max(res["primal"], res["dual"], res["gap"]) <= tol
    scale = max(1.0, abs(lp.optimal_objective))
    assert abs(h.objective - lp.optimal_objective) <= 1e-5 * scale
    print(f"{precision}: halpern {h.iterations} iterations, reference operator {r.iterations}")


def test_repeatable_bit_for_bit():
    lp = lpgen.uniform_planted(300, 700, 6, seed=5)
    a = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-7))
    b = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-7))
    assert a.iterations == b.iterations
    assert np.array_equal(a.col_value, b.col_value)


def test_certificates():
    rng = np.random.default_rng(7)
    inf = lpgen.make_infeasible(lpgen.uniform_planted(60, 150, 4, seed=1), rng)
    unb = lpgen.make_unbounded(lpgen.uniform_planted(60, 150, 4, seed=2), rng)
    s = P.solve_pdhg(inf, _opts(pdhg_tolerance=1e-6, iteration_limit=200000))
    assert s.status == "infeasible", s.message
    assert farkas_ok(inf, s.farkas_dual)[0]
    s = P.solve_pdhg(unb, _opts(pdhg_tolerance=1e-6, iteration_limit=200000))
    assert s.status == "unbounded", s.message
    assert ray_ok(unb, s.primal_ray)[0]


def test_batched_engine_with_the_halpern_operator():
    """Batched: every feasible LP meets the request, certificates pass the reference's
    checkers, and each answer is the same alone, in the mix and when served in chunks."""
    rng = np.random.default_rng(9)
    lps = lpgen.uneven_batch(count=24, m_lo=50, m_hi=600, infeasible_fraction=0.2, seed=13)
    lps.append(lpgen.make_unbounded(lpgen.uniform_planted(80, 200, 4, seed=3), rng))
    opts = _opts(pdhg_tolerance=1e-6, pdhg_stop_rule="relative_kkt", iteration_limit=200000)
    sols = P.batch_solve(lps, opts)
    for lp, s in zip(lps, sols):
        if lp.farkas_star is not None:
            assert s.status == "infeasible", (lp.name, s.status, s.message)
            assert farkas_ok(lp, s.farkas_dual)[0], lp.name
        elif lp.ray_star is not None:
            # the batched engine claims unboundedness only with a feasible point; else the
            # certified ray comes back alone
            assert s.status in ("unbounded", "infeasible_or_unbounded"), (lp.name, s.status,
                                                                          s.message)
            assert ray_ok(lp, s.primal_ray)[0], lp.name
        else:
            assert s.status in ("optimal", "feasible"), (lp.name, s.status, s.message)
            r = oracle.oracle_evaluate(lp, s.col_value, -s.row_dual)
            assert max(r["primal"], r["dual"], r["gap"]) <= 1e-6, (lp.name, r)
    alone = P.batch_solve([lps[5]], opts)[0]
    assert alone.iterations == sols[5].iterations
    assert np.array_equal(alone.col_value, sols[5].col_value)
    with P.Server(chunk_attempts=100) as srv:
        chunked = srv.solve_all(lps[:8], opts)
    for a, b in zip(chunked, sols[:8]):
        assert a.status == b.status and a.iterations == b.iterations
        assert np.array_equal(a.col_value, b.col_value)
