"""The reference's own instances on the GPU.

* Netlib (the reference tree's data/netlib/*.mps, read by the reference's MPS reader into
  tests/golden/netlib.npz): at pdhg_tolerance 1e-8 under the reference's stop rule, every LP
  the reference's solve_pdhg solves comes back optimal with its objective within 1e-6 of the
  published optimum (data/netlib/reference.json), in FP64 with both operators and in
  FP32-mixed. share2b, where the reference's PDHG stops at its iteration limit, must not be
  claimed optimal unless it meets that bar too.
* The reference's cross-engine gate (tests/unit/test_pdhg.cpp:178-222): its 120 generated
  instances (tests/golden/kkt_fuzz_120.npz) at pdhg_tolerance 1e-9; every instance both the
  GPU and the reference solve optimally must agree with the analytic optimum to 1e-6, and more
  than 60 must be compared -- the gate's own bar -- on the single-LP path and through the
  batched engine.
"""
import pytest

from sih26_b200 import pdhg as P
from tests.cases import kkt_fuzz_cases, netlib_cases

pytestmark = pytest.mark.gpu

VARIANTS = [("fp64", "reference"), ("fp64", "halpern"), ("mixed", "halpern")]


@pytest.mark.parametrize("precision,algorithm", VARIANTS)
@pytest.mark.parametrize("case", netlib_cases(), ids=lambda c: c[0].name)
def test_netlib_published_optima(case, precision, algorithm):
    lp, published, ref_status, _ = case
    if algorithm == "reference" and lp.name in ("stocfor1", "israel", "share2b"):
        pytest.skip("the reference operator needs 0.5-1M iterations here; run with Halpern")
    s = P.solve_pdhg(lp, P.Options(pdhg_tolerance=1e-8, iteration_limit=1000000,
                                   pdhg_precision=precision, pdhg_algorithm=algorithm))
    ok = abs(s.objective - published) <= 1e-6 * max(1.0, abs(published))
    if ref_status == "optimal":
        assert s.status == "optimal", (lp.name, s.status, s.message)
        assert ok, (lp.name, s.objective, published)
    else:
        assert s.status in ("optimal", "iteration_limit"), (lp.name, s.status)
        if s.status == "optimal":
            assert ok, (lp.name, s.objective, published)


def _agree(cases, sols):
    compared = disagreed = 0
    worst = 0.0
    for (lp, ref_status, _), s in zip(cases, sols):
        if ref_status != "optimal" or s.status != "optimal":
            continue
        compared += 1
        rel = abs(s.objective - lp.optimal_objective) / max(1.0, abs(lp.optimal_objective))
        worst = max(worst, rel)
        disagreed += rel > 1e-6
    return compared, disagreed, worst


@pytest.mark.parametrize("algorithm", ["reference", "halpern"])
def test_cross_engine_gate_single_lp(algorithm):
    cases = kkt_fuzz_cases()
    opts = P.Options(pdhg_tolerance=1e-9, iteration_limit=1000000, pdhg_algorithm=algorithm)
    sols = [P.solve_pdhg(lp, opts) for lp, _, _ in cases]
    compared, disagreed, worst = _agree(cases, sols)
    assert disagreed == 0, worst
    assert compared > 60, compared


def test_cross_engine_gate_batched():
    cases = kkt_fuzz_cases()
    sols = P.batch_solve([lp for lp, _, _ in cases],
                         P.Options(pdhg_tolerance=1e-9, iteration_limit=1000000,
                                   pdhg_algorithm="halpern"))
    compared, disagreed, worst = _agree(cases, sols)
    assert disagreed == 0, worst
    assert compared > 60, compared
