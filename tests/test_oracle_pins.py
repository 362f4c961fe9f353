"""Pins the oracle (oracle/pdhg_oracle.c) to the reference before anything is checked
against it.

* against tests/golden/reference_pdhg.json, recorded from the reference's own solve_pdhg
  (runs anywhere);
* against the reference built from its sources (oracle/_ref), bit for bit, when that build
  exists (this container);
* against the known answers of the reference's unit tests (tests/unit/test_pdhg.cpp,
  tests/unit/test_gpu.cpp).
"""
import json
import math
import os

import numpy as np
import pytest

import oracle
from cases import generated_cases, hand_cases
from sih26_b200 import lpgen

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_pdhg.json")


def _cases_by_name():
    d = {n: lp for n, lp, _ in hand_cases()}
    d.update(dict(generated_cases()))
    return d


def test_oracle_reproduces_reference_fixture_exactly():
    golden = json.load(open(GOLDEN))
    cases = _cases_by_name()
    assert len(golden["cases"]) >= 40
    for rec in golden["cases"]:
        lp = cases[rec["case"]]
        r = oracle.oracle_solve(lp, tolerance=rec["opt_tolerance"],
                                iteration_limit=rec["opt_iteration_limit"],
                                restart=rec["opt_restart"],
                                stop_at_request=rec["opt_stop_at_request"])
        key = (rec["case"], rec["options"])
        assert r.status == rec["status"], key
        assert r.iterations == rec["iterations"], key
        # same operations in the same order: the objective is bit-identical
        assert r.objective == rec["objective"], key
        assert float(np.sum(r.col_value)) == rec["x_sum"], key
        if rec["col_value"] is not None:
            assert r.col_value.tolist() == rec["col_value"], key


@pytest.mark.parametrize("name,lp,expected", hand_cases())
def test_oracle_meets_reference_unit_test_answers(name, lp, expected):
    r = oracle.oracle_solve(lp, tolerance=1e-8, iteration_limit=200000)
    assert r.status == "optimal", name
    if expected is not None:
        assert abs(r.objective - expected) <= 1e-5 * max(1.0, abs(expected)), name
    if name == "original_sense":  # test_pdhg.cpp:136-137
        assert abs(r.col_value[0] - 2.0) < 1e-4 and abs(r.col_value[1] - 6.0) < 1e-4
    if name == "minimises_a_sum":  # test_pdhg.cpp:248-263, the step-size collapse guard
        assert r.iterations < 500
    if name == "blend":  # test_pdhg.cpp:474-488 (the polished solve() value)
        assert abs(r.objective - 214.14594594594595) < 1e-4


def test_oracle_iteration_limit_is_honest():
    """test_pdhg.cpp:148-157: a 20-iteration run claims nothing."""
    lp = lpgen.from_dense([[1, 1]], [2], [math.inf], [1, 1])
    r = oracle.oracle_solve(lp, tolerance=1e-12, iteration_limit=20)
    assert r.status != "optimal"
    assert math.isinf(r.dual_bound)


def test_planted_optimum_is_found():
    lp = lpgen.uniform_planted(200, 500, 5, seed=7)
    r = oracle.oracle_solve(lp, tolerance=1e-8)
    assert r.status == "optimal"
    assert abs(r.objective - lp.optimal_objective) <= 1e-6 * max(1.0, abs(lp.optimal_objective))


needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference build (make -C oracle ref) not present")


@needs_ref
def test_scaling_and_norm_bit_identical_to_reference():
    for _, lp in generated_cases():
        mc = lp.cost.copy()
        a, b = oracle.oracle_scaling(lp, mc), oracle.ref_scaling(lp, mc)
        for k in a:
            assert np.array_equal(a[k], b[k]), k
        assert oracle.oracle_spectral_norm(lp, 30, 1) == oracle.ref_spectral_norm(lp, 30, 1)


@needs_ref
@pytest.mark.parametrize("seed", [11, 12])
def test_oracle_bit_identical_to_reference_build(seed):
    lp = lpgen.uniform_planted(120, 300, 6, seed=seed)
    for opts in (dict(tolerance=1e-8), dict(tolerance=1e-5, stop_at_request=True),
                 dict(tolerance=1e-7, restart=False)):
        a = oracle.oracle_solve(lp, **opts)
        b = oracle.ref_solve(lp, **opts)
        assert (a.status, a.iterations) == (b.status, b.iterations)
        assert np.array_equal(a.col_value, b.col_value)
        assert np.array_equal(a.row_dual, b.row_dual)
        assert np.array_equal(a.col_dual, b.col_dual)


NETLIB = "/root/reference/data/netlib"


@needs_ref
@pytest.mark.skipif(not os.path.isdir(NETLIB), reason="reference Netlib files not present")
@pytest.mark.parametrize("name", ["afiro", "sc50a", "sc50b", "blend"])
def test_oracle_on_netlib_matches_reference(name):
    lp = oracle.ref_read_model(os.path.join(NETLIB, name + ".mps"))
    a = oracle.oracle_solve(lp, tolerance=1e-8, iteration_limit=200000)
    b = oracle.ref_solve(lp, tolerance=1e-8, iteration_limit=200000)
    assert (a.status, a.iterations) == (b.status, b.iterations)
    assert a.objective == b.objective
    ref = json.load(open(os.path.join(NETLIB, "reference.json")))["instances"][name]
    assert abs(a.objective - ref["published_optimal"]) <= 1e-6 * abs(ref["published_optimal"])


def test_oracle_steps_meet_the_reference_gpu_slot_known_answers():
    """The known answers of the reference's GPU-slot tests, on the oracle's own primal step and
    CSC products (the code its solve runs): the 4-coordinate primal step with a box, a free, a
    lower-bounded and an interior column (tests/unit/test_gpu.cpp:107-140), and the 2 x 3 CSC
    product in both orientations (:142-177). The reference allows 1e-12; every value here is
    exact in binary, so equality is required."""
    inf = math.inf
    x_next, extrapolated = oracle.oracle_primal_step(
        0.5, x=[2.0, 0.0, -4.0, 0.5], cost=[1.0, -2.0, 2.0, 3.0], at_y=[0.0, 1.0, 0.0, 0.0],
        lower=[-1.0, 0.0, -inf, 0.0], upper=[1.0, 2.0, inf, inf])
    assert x_next.tolist() == [1.0, 0.5, -5.0, 0.0]
    assert extrapolated.tolist() == [0.0, 1.0, -6.0, -0.5]

    cs, ri, val = [0, 1, 2, 4], [0, 1, 0, 1], [1.0, 3.0, 2.0, 4.0]  # [[1 0 2] [0 3 4]]
    assert oracle.oracle_csc_multiply(2, cs, ri, val, [1.0, 2.0, 3.0]).tolist() == [7.0, 18.0]
    assert oracle.oracle_csc_transpose_multiply(cs, ri, val, [2.0, 5.0]).tolist() == [2.0, 15.0,
                                                                                       24.0]
    # an absent bound given as a large finite value (|v| >= 1e30) projects like an infinite one
    x_next, _ = oracle.oracle_primal_step(1.0, x=[0.0, 0.0], cost=[1e3, -1e3], at_y=[0.0, 0.0],
                                          lower=[-1e30, -1e31], upper=[1e30, 2e30])
    assert x_next.tolist() == [-1e3, 1e3]


def test_stop_at_request_on_adlittle_as_the_reference_test_pins_it():
    """tests/unit/test_pdhg.cpp:339-381 on the oracle: adlittle (data/netlib, read by the
    reference's reader) at a 1e-4 request. The honest run is optimal; with pdhg_stop_at_request
    the loop stops earlier, on a point reported feasible (it does not meet the absolute
    standard), primal-feasible to 1e-7 and at the honest objective to 1e-3 relative. The
    reference test runs the whole solve(), presolve included, and its recorded counts (132,520
    and 192,080, bench/results/pdhg-stop-at-request-f18d4b0.csv, pdhg-79ec7f7.csv) are of the
    presolved model; on the model as read, solve_pdhg itself takes 72,400 and 209,160, and the
    oracle must equal the reference build there iteration for iteration."""
    from cases import netlib_cases

    lp = next(c[0] for c in netlib_cases() if c[0].name == "adlittle")
    honest = oracle.oracle_solve(lp, tolerance=1e-4, iteration_limit=1000000)
    cheap = oracle.oracle_solve(lp, tolerance=1e-4, iteration_limit=1000000,
                                stop_at_request=True)
    assert honest.status == "optimal" and cheap.status == "feasible"
    assert cheap.iterations < honest.iterations
    assert (cheap.iterations, honest.iterations) == (72400, 209160)
    assert cheap.residuals["absolute_primal"] <= 1e-7
    assert abs(cheap.objective - honest.objective) <= 1e-3 * max(1.0, abs(honest.objective))
    if oracle.ref_available():
        for mine, sar in ((honest, False), (cheap, True)):
            ref = oracle.ref_solve(lp, tolerance=1e-4, iteration_limit=1000000,
                                   stop_at_request=sar)
            assert (ref.status, ref.iterations, ref.objective) == (mine.status, mine.iterations,
                                                                   mine.objective)
            assert np.array_equal(ref.col_value, mine.col_value)
