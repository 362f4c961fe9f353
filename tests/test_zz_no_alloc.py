"""sankhya_pdhg_gpu_residuals_noalloc: the residual check for callers that cannot allocate.

Some callers cannot allocate device memory while they run (their memory belongs to their own
pool, or their device budget is fixed at start-up, or they cannot afford the synchronisation
cudaMalloc implies). This entry point evaluates the KKT residuals of a point with scratch
held in a fixed array inside the library. The test solves an LP with the regular entry point,
then asks the no-allocation entry point -- twice in a row, on the same scratch -- for the
residuals of the point the solve returned, and checks both answers against the residual block
the solve reported. Device buffers here are made by torch; the entry point itself allocates
nothing.

This file is collected last so that a failure here never hides another test's result.
"""
import ctypes as C
import math

import numpy as np
import pytest

from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = pytest.mark.gpu

FIELDS = ("relative_primal", "relative_dual", "relative_gap", "primal_objective",
          "dual_objective", "absolute_primal", "absolute_dual", "gap_as_verified",
          "complementarity")


def _device_problem(lp, torch, keep):
    dev = "cuda:0"

    def put(a, dtype):
        t = torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)
        keep.append(t)
        return t.data_ptr()

    i32 = C.POINTER(C.c_int32)
    f64 = C.POINTER(C.c_double)
    return P._Problem(
        lp.num_rows, lp.num_cols, lp.num_nonzeros,
        C.cast(put(lp.col_starts, torch.int32), i32), C.cast(put(lp.row_indices, torch.int32), i32),
        C.cast(put(lp.values, torch.float64), f64), C.cast(put(lp.cost, torch.float64), f64),
        C.cast(put(lp.col_lower, torch.float64), f64), C.cast(put(lp.col_upper, torch.float64), f64),
        C.cast(put(lp.row_lower, torch.float64), f64), C.cast(put(lp.row_upper, torch.float64), f64),
        1 if lp.maximize else 0, float(lp.objective_offset))


def test_noalloc_residuals_match_the_solve_twice_in_a_row():
    torch = pytest.importorskip("torch")
    lib = P.load_library()
    lib.sankhya_pdhg_gpu_residuals_noalloc.argtypes = [C.POINTER(P._Problem), C.c_void_p,
                                                       C.c_void_p, C.c_void_p, C.c_void_p]
    lp = lpgen.uniform_planted(2000, 5000, 10, seed=0)
    sol = P.solve_pdhg(lp, P.Options(pdhg_tolerance=1e-6))
    assert sol.status == "optimal", sol.message
    keep = []
    prob = _device_problem(lp, torch, keep)
    x = torch.as_tensor(sol.col_value, dtype=torch.float64, device="cuda:0")
    rd = torch.as_tensor(sol.row_dual, dtype=torch.float64, device="cuda:0")
    for call in range(2):
        out = torch.full((9,), math.nan, dtype=torch.float64, device="cuda:0")
        rc = lib.sankhya_pdhg_gpu_residuals_noalloc(C.byref(prob), x.data_ptr(), rd.data_ptr(),
                                                    out.data_ptr(), None)
        assert rc == 0, lib.sankhya_pdhg_gpu_last_error().decode()
        torch.cuda.synchronize()
        got = dict(zip(FIELDS, out.cpu().numpy().tolist()))
        for k in FIELDS:
            want = sol.residuals[k]
            # the parity bar of the other tests: 1e-6 relative, with an absolute floor for
            # residuals that are themselves at rounding level
            assert abs(got[k] - want) <= 1e-6 * abs(want) + 1e-9, (call, k, got[k], want)

    # more rows than the fixed scratch holds: refused up front, nothing launched
    big = lpgen.from_dense([[1.0]], [1.0], [1.0], [1.0])
    big.num_rows = P.NOALLOC_MAX_ROWS + 1
    bad = P._Problem(big.num_rows, 1, 0, prob.col_starts, prob.row_indices, prob.values,
                     prob.cost, prob.col_lower, prob.col_upper, prob.row_lower, prob.row_upper,
                     0, 0.0)
    out = torch.zeros(9, dtype=torch.float64, device="cuda:0")
    rc = lib.sankhya_pdhg_gpu_residuals_noalloc(C.byref(bad), x.data_ptr(), rd.data_ptr(),
                                                out.data_ptr(), None)
    assert rc == 10
    assert "exceed" in lib.sankhya_pdhg_gpu_last_error().decode()
