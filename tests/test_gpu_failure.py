"""The bounded grid barrier's give-up path, made to run on purpose.

Every spin of the iteration kernels' grid barrier gives up after a time limit, records an
error word and returns, so a launch in which a block never arrives ends with
SANKHYA_GPU_DEVICE_TIMEOUT (the status vocabulary of include/sankhya/gpu_runtime.hpp:19-30
plus this library's timeout) instead of hanging the GPU. The test switches on the library's
fault injection (SANKHYA_PDHG_TEST_BARRIER_FAULT: the last block of the iteration kernel stays
away from its first barrier, the others give up after 200 ms), checks the status and the
message, and then checks that the next solve on the same context is normal again. Nothing
faults: every wait is bounded and every access stays in bounds.
"""
import pytest

from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = pytest.mark.gpu

DEVICE_TIMEOUT = 11


@pytest.mark.parametrize("precision,algorithm", [("fp64", "reference"), ("mixed", "halpern"),
                                                 ("fp64", "halpern")])
def test_barrier_gives_up_and_the_next_solve_is_normal(monkeypatch, precision, algorithm):
    lp = lpgen.uniform_planted(2000, 5000, 10, seed=5)  # several blocks, so some must wait
    opts = P.Options(pdhg_tolerance=1e-6, pdhg_precision=precision, pdhg_algorithm=algorithm,
                     pdhg_stop_rule="relative_kkt")
    monkeypatch.setenv("SANKHYA_PDHG_TEST_BARRIER_FAULT", "200")
    with pytest.raises(P.GpuError) as err:
        P.solve_pdhg(lp, opts)
    assert err.value.code == DEVICE_TIMEOUT, str(err.value)
    assert "grid barrier timed out" in str(err.value)
    monkeypatch.delenv("SANKHYA_PDHG_TEST_BARRIER_FAULT")
    s = P.solve_pdhg(lp, opts)
    assert s.status in ("optimal", "feasible"), s.message
    r = s.residuals
    assert max(r["relative_primal"], r["relative_dual"], r["relative_gap"]) <= 1e-6
