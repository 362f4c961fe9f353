"""Infeasibility and unboundedness on the GPU: every certificate the CUDA path reports passes
the reference's own checkers (src/core/certificate.cpp:29-218), on the single-LP path in both
precisions and in the batched engine. The reference's CPU PDHG never certifies either case
(src/pdhg/pdhg.cpp:697-707 ends such LPs at the iteration or time limit); these tests hold the
GPU path to the checker instead."""
import numpy as np
import pytest

from certs import farkas_ok, ray_ok
from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = pytest.mark.gpu

INF = float("inf")


def _opts(**kw):
    o = P.Options(pdhg_tolerance=1e-6, iteration_limit=200000)
    for k, v in kw.items():
        o.set(k, v)
    return o


def _infeasible(seed, m=60, n=150):
    rng = np.random.default_rng(100 + seed)
    return lpgen.make_infeasible(lpgen.uniform_planted(m, n, 4, seed=seed), rng)


def _unbounded(seed, m=60, n=150):
    rng = np.random.default_rng(200 + seed)
    return lpgen.make_unbounded(lpgen.uniform_planted(m, n, 4, seed=seed), rng)


HAND_INFEASIBLE = lpgen.from_dense([[1, 1]], [3], [3], [1, 1], col_upper=[1.0, 1.0],
                                   name="sum_of_two_unit_boxes_is_three")
HAND_UNBOUNDED = lpgen.from_dense([[1, -1]], [0], [0], [-1, -1], name="equal_pair_runs_off")
HAND_UNBOUNDED_MAX = lpgen.from_dense([[1, -1], [1, 0]], [0, 1], [0, INF], [1, 1],
                                      maximize=True, name="maximise_an_equal_pair")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("lp", [HAND_INFEASIBLE, _infeasible(1), _infeasible(2)],
                         ids=lambda lp: lp.name)
def test_infeasible_lp_returns_a_checked_farkas_certificate(lp, precision):
    s = P.solve_pdhg(lp, _opts(pdhg_precision=precision))
    assert s.status == "infeasible", (lp.name, s.status, s.message)
    assert s.farkas_dual is not None and s.farkas_dual.shape == (lp.num_rows,)
    ok, why = farkas_ok(lp, s.farkas_dual)
    assert ok, (lp.name, why)
    assert "Farkas" in s.message


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("lp", [HAND_UNBOUNDED, HAND_UNBOUNDED_MAX, _unbounded(1), _unbounded(2)],
                         ids=lambda lp: lp.name)
def test_unbounded_lp_returns_a_checked_primal_ray(lp, precision):
    s = P.solve_pdhg(lp, _opts(pdhg_precision=precision))
    assert s.status == "unbounded", (lp.name, s.status, s.message)
    assert s.primal_ray is not None and s.primal_ray.shape == (lp.num_cols,)
    ok, why = ray_ok(lp, s.primal_ray)
    assert ok, (lp.name, why)
    # the ray starts from a feasible point (a zero-cost solve of the constraints found it)
    assert s.primal_infeasibility <= 1e-7, (lp.name, s.primal_infeasibility)
    assert "feasible point" in s.message
    if lp.ray_star is not None:  # the planted direction, up to scale
        r = s.primal_ray / np.max(np.abs(s.primal_ray))
        assert np.allclose(r, lp.ray_star / np.max(np.abs(lp.ray_star)), atol=1e-6)


def test_detection_off_runs_to_the_limit_like_the_reference():
    s = P.solve_pdhg(HAND_INFEASIBLE, _opts(pdhg_detect_infeasibility=False, iteration_limit=3000))
    assert s.status == "iteration_limit", s.status
    assert s.farkas_dual is None


def test_batched_engine_certifies_both_kinds_next_to_feasible_lps():
    rng = np.random.default_rng(5)
    lps = []
    for k in range(12):
        base = lpgen.uniform_planted(50 + 10 * k, 120 + 20 * k, 4, seed=30 + k)
        if k % 3 == 1:
            base = lpgen.make_infeasible(base, rng)
        elif k % 3 == 2:
            base = lpgen.make_unbounded(base, rng)
        lps.append(base)
    sols = P.batch_solve(lps, _opts(pdhg_stop_rule="relative_kkt"))
    for k, (lp, s) in enumerate(zip(lps, sols)):
        if k % 3 == 0:
            assert s.status in ("optimal", "feasible"), (lp.name, s.status, s.message)
            assert abs(s.objective - lp.optimal_objective) <= 1e-4 * max(1.0, abs(lp.optimal_objective))
        elif k % 3 == 1:
            assert s.status == "infeasible", (lp.name, s.status, s.message)
            ok, why = farkas_ok(lp, s.farkas_dual)
            assert ok, (lp.name, why)
        else:
            # the batched engine claims unboundedness only when its point is feasible too;
            # otherwise the certified ray comes back alone
            assert s.status in ("unbounded", "infeasible_or_unbounded"), (lp.name, s.status,
                                                                          s.message)
            ok, why = ray_ok(lp, s.primal_ray)
            assert ok, (lp.name, why)
            if s.status == "unbounded":
                assert s.primal_infeasibility <= 1e-7, (lp.name, s.primal_infeasibility)
