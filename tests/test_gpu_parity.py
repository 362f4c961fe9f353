"""Parity of the CUDA PDHG path with the reference (golden fixture) and the oracle.

Bar (restated from the reference's own checks): same status; objective within 1e-6 relative
(test_pdhg.cpp:178-222 uses 1e-6 against the simplex); the returned point's unscaled
residuals, recomputed by the oracle from the point itself, meet the request; the same
active-bound pattern as the oracle's point; and the reference's unit-test answers.
"""
import json
import math
import os

import numpy as np
import pytest

import oracle
from cases import generated_cases, hand_cases
from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_pdhg.json")


def _opts(**kw):
    o = P.Options()
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


@pytest.mark.parametrize("name,lp,expected", hand_cases())
def test_reference_unit_test_answers(name, lp, expected):
    s = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-8, iteration_limit=200000))
    assert s.status == "optimal", (name, s.message)
    assert s.algorithm == "pdhg-gpu"
    if expected is not None:
        assert abs(s.objective - expected) <= 1e-6 * max(1.0, abs(expected)), name
    if name == "original_sense":
        assert abs(s.col_value[0] - 2.0) < 1e-4 and abs(s.col_value[1] - 6.0) < 1e-4
    if name == "minimises_a_sum":
        assert s.iterations < 500  # the step-size collapse guard, test_pdhg.cpp:248-263
    if name == "blend":
        assert abs(s.objective - 214.14594594594595) < 1e-4
    if name == "large_rhs":  # optimal is never claimed on a point that fails verification
        assert s.primal_infeasibility <= 1e-7


def test_matches_reference_fixture():
    """Every fixture record: same status, objective within 1e-6, iteration count close.

    The GPU sums in a different order, so its trajectory drifts from the reference's by
    rounding; restarts and the stopping test can then trigger a few evaluations apart. Under
    pdhg_stop_at_request both `feasible` and `optimal` mean "stopped on the request"; which
    one is reported depends on whether the stopping point also happens to meet the absolute
    standard, and on a borderline point that turns on rounding. That interchange is the one
    status difference accepted, and it is counted. The GPU may converge faster than the
    reference; it may not be more than 50 % slower."""
    golden = json.load(open(GOLDEN))
    cases = {n: lp for n, lp, _ in hand_cases()}
    cases.update(dict(generated_cases()))
    worst_slowdown = 0.0
    mismatches, interchanges, lines = [], 0, []
    for rec in golden["cases"]:
        lp = cases[rec["case"]]
        s = P.solve_pdhg(lp, _opts(pdhg_tolerance=rec["opt_tolerance"],
                                   iteration_limit=rec["opt_iteration_limit"],
                                   pdhg_restart=rec["opt_restart"],
                                   pdhg_stop_at_request=rec["opt_stop_at_request"]))
        key = (rec["case"], rec["options"])
        lines.append(f"{key}: ref {rec['status']} {rec['iterations']} / gpu {s.status} {s.iterations}")
        if s.status != rec["status"]:
            if rec["opt_stop_at_request"] and {s.status, rec["status"]} == {"feasible", "optimal"}:
                interchanges += 1
            else:
                mismatches.append((key, rec["status"], s.status, s.message))
                continue
        if rec["status"] in ("optimal", "feasible"):
            scale = max(1.0, abs(rec["objective"]))
            assert abs(s.objective - rec["objective"]) <= 1e-6 * scale, key
            assert s.primal_infeasibility <= 1e-7, key
        else:
            assert s.iterations == rec["iterations"], key  # the limit itself
            assert math.isinf(s.dual_bound)
        ref_it = rec["iterations"]
        worst_slowdown = max(worst_slowdown, (s.iterations - ref_it) / max(ref_it, 40))
    print("\n".join(lines))
    print(f"feasible/optimal interchanges under stop_at_request: {interchanges}; "
          f"worst slowdown {worst_slowdown:.2f}")
    assert not mismatches, mismatches
    assert interchanges <= 3
    assert worst_slowdown <= 0.5


@pytest.mark.parametrize("name,lp", generated_cases())
def test_generated_against_oracle(name, lp):
    tol = 1e-8
    s = P.solve_pdhg(lp, _opts(pdhg_tolerance=tol))
    o = oracle.oracle_solve(lp, tolerance=tol)
    assert s.status == o.status == "optimal", s.message
    scale = max(1.0, abs(o.objective))
    assert abs(s.objective - o.objective) <= 1e-6 * scale
    assert abs(s.objective - lp.optimal_objective) <= 1e-6 * scale
    # residuals recomputed by the oracle from the returned point alone
    r = oracle.oracle_evaluate(lp, s.col_value, _y_pdhg_sign(lp, s))
    assert max(r["primal"], r["dual"], r["gap"]) <= tol
    assert r["absolute_primal"] <= 1e-7 and r["gap_as_verified"] <= 1e-9
    assert np.array_equal(_pattern(lp, s.col_value), _pattern(lp, o.col_value))
    assert abs(s.iterations - o.iterations) <= max(80, 0.25 * o.iterations)


def test_stop_at_request_gives_the_cheap_answer():
    lp = lpgen.uniform_planted(200, 500, 5, seed=7)
    honest = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-4))
    cheap = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-4, pdhg_stop_at_request=True))
    assert honest.status == "optimal"
    assert cheap.status in ("feasible", "optimal")
    assert cheap.iterations <= honest.iterations
    assert "pdhg_stop_at_request" in cheap.message or cheap.status == "optimal"
    assert cheap.primal_infeasibility <= 1e-7


def test_iteration_limit_claims_nothing():
    lp = lpgen.from_dense([[1, 1]], [2], [math.inf], [1, 1])
    s = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-12, iteration_limit=20))
    assert s.status == "iteration_limit" and s.iterations == 20
    assert math.isinf(s.dual_bound) and s.message


def test_repeatable_bit_for_bit():
    lp = lpgen.uniform_planted(300, 700, 6, seed=5)
    a = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-7))
    b = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-7))
    assert a.iterations == b.iterations
    assert np.array_equal(a.col_value, b.col_value)
    assert np.array_equal(a.row_dual, b.row_dual)


def test_time_limit_is_honoured():
    lp = lpgen.uniform_planted(2000, 5000, 10, seed=3)
    s = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-14, time_limit=0.5, iteration_limit=10**7))
    assert s.status == "time_limit"
    assert s.solve_seconds < 5.0


@pytest.mark.slow
def test_single_lp_2000x5000_against_oracle():
    """The 2,000 x 5,000 planted LP with 10 nonzeros per column, solved to 1e-6."""
    lp = lpgen.uniform_planted(2000, 5000, 10, seed=0)
    s = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-6))
    o = oracle.oracle_solve(lp, tolerance=1e-6)
    assert s.status == o.status == "optimal"
    scale = max(1.0, abs(lp.optimal_objective))
    assert abs(s.objective - lp.optimal_objective) <= 1e-6 * scale
    assert abs(s.objective - o.objective) <= 1e-6 * scale
    assert np.array_equal(_pattern(lp, s.col_value), _pattern(lp, o.col_value))


@pytest.mark.parametrize("rule", ["relative_kkt", "reference"])
def test_mixed_precision_against_oracle(rule):
    """FP32 iterates with FP64 reductions, then the FP64 polish when the request needs it."""
    lp = lpgen.uniform_planted(2000, 5000, 10, seed=0)
    tol = 1e-6
    s = P.solve_pdhg(lp, _opts(pdhg_tolerance=tol, pdhg_precision="mixed", pdhg_stop_rule=rule))
    assert s.status in ("optimal", "feasible"), s.message
    assert s.fp32_iterations > 0
    r = oracle.oracle_evaluate(lp, s.col_value, _y_pdhg_sign(lp, s))
    assert max(r["primal"], r["dual"], r["gap"]) <= tol
    scale = max(1.0, abs(lp.optimal_objective))
    assert abs(s.objective - lp.optimal_objective) <= 1e-6 * scale
    if rule == "reference":
        assert s.status == "optimal"
        assert s.iterations > s.fp32_iterations  # the FP64 polish ran
        o = oracle.oracle_solve(lp, tolerance=tol)
        assert np.array_equal(_pattern(lp, s.col_value), _pattern(lp, o.col_value))


def test_mixed_hand_over_keeps_the_restart_state():
    """An early switch hands the FP32 level's whole restart state to FP64: the solve goes on
    and meets the request."""
    lp = lpgen.uniform_planted(2000, 5000, 10, seed=0)
    tol = 1e-6
    s = P.solve_pdhg(lp, _opts(pdhg_tolerance=tol, pdhg_precision="mixed",
                               pdhg_stop_rule="relative_kkt", pdhg_mixed_switch_tolerance=1e-3))
    assert s.status in ("optimal", "feasible"), s.message
    assert 0 < s.fp32_iterations < s.iterations
    r = oracle.oracle_evaluate(lp, s.col_value, _y_pdhg_sign(lp, s))
    assert max(r["primal"], r["dual"], r["gap"]) <= tol


def test_mixed_reaches_a_tolerance_below_plain_fp32():
    """FP32 deltas about an FP64 anchor have no FP32 floor at 1e-8 (plain FP32 iterates stall
    around 1e-5 to 1e-6 relative KKT); the answer meets the request either way."""
    lp = lpgen.uniform_planted(2000, 5000, 10, seed=0)
    tol = 1e-8
    s = P.solve_pdhg(lp, _opts(pdhg_tolerance=tol, pdhg_precision="mixed",
                               pdhg_stop_rule="relative_kkt"))
    assert s.status in ("optimal", "feasible"), s.message
    r = oracle.oracle_evaluate(lp, s.col_value, _y_pdhg_sign(lp, s))
    assert max(r["primal"], r["dual"], r["gap"]) <= tol
    print("fp32 iterations", s.fp32_iterations, "of", s.iterations)


@pytest.mark.slow
def test_block_angular_full_size_mixed_to_1e6():
    """The blending-style block-angular LP at full size (64 blocks of 4,000 x 10,000 plus 2,000
    linking rows touching 2 % of all columns: 258,000 x 640,000, ~30.7M nonzeros, 30 % '<='
    rows), FP32-mixed with the FP64 polish when needed, to relative KKT 1e-6. The oracle is too
    slow at this size, so the checks are the size-independent ones: the residuals recomputed
    by the oracle's evaluate from the returned point meet the request, and the objective
    matches the planted optimum to the accuracy such a point carries."""
    lp = lpgen.block_angular_planted(seed=2)
    assert lp.num_rows == 258_000 and lp.num_cols == 640_000
    for algorithm in ("halpern", "reference"):
        s = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-6, pdhg_stop_rule="relative_kkt",
                                   pdhg_precision="mixed", pdhg_algorithm=algorithm,
                                   iteration_limit=400000))
        assert s.status in ("optimal", "feasible"), (algorithm, s.message)
        r = oracle.oracle_evaluate(lp, s.col_value, _y_pdhg_sign(lp, s))
        assert max(r["primal"], r["dual"], r["gap"]) <= 1e-6, (algorithm, r)
        scale = max(1.0, abs(lp.optimal_objective))
        assert abs(s.objective - lp.optimal_objective) <= 1e-5 * scale, algorithm
        print(f"{algorithm}: {s.iterations} iterations ({s.fp32_iterations} FP32), "
              f"{s.device_seconds:.2f} s on the device")


def test_device_primal_infeasibility_matches_the_host_figure():
    """Solution::recompute_quality's primal_infeasibility (src/core/model.cpp:228-283), which the
    library now computes on the device for every answer, against the same figure on the host."""
    lps = [lp for _, lp in generated_cases()] + [lp for _, lp, _ in hand_cases()]
    for lp in lps:
        s = P.solve_pdhg(lp, _opts(pdhg_tolerance=1e-4, iteration_limit=2000))
        host = P.primal_infeasibility_host(lp, s.col_value)
        scale = max(1.0, float(np.max(np.abs(s.col_value))) if s.col_value.size else 1.0)
        assert abs(s.primal_infeasibility - host) <= 1e-9 * scale, (lp.name, s.primal_infeasibility, host)
    sols = P.batch_solve(lps[:4], _opts(pdhg_tolerance=1e-4, iteration_limit=2000))
    for lp, s in zip(lps[:4], sols):
        host = P.primal_infeasibility_host(lp, s.col_value)
        assert abs(s.primal_infeasibility - host) <= 1e-9 * max(1.0, float(np.max(np.abs(s.col_value))))
