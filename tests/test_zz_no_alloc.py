"""sankhya_pdhg_gpu_residuals_noalloc: the residual check for callers that cannot allocate.

Some callers cannot allocate device memory while they run: their device memory belongs to
their own pool or arena, their device budget is fixed at start-up, or they cannot afford the
device-wide synchronisation cudaMalloc and cudaFree imply. This entry point evaluates the
unscaled KKT residuals of a point (the residual block of src/pdhg/pdhg.cpp:143-263) with its
scratch held in a fixed array inside the library.

The tests hand it LPs with every row and bound kind in both senses (>=, <= and range rows,
free and fixed columns, maximisation, an inequality-rich block-angular LP) and check, on two
calls in a row on the same scratch and on a non-default stream:

* all nine fields against the oracle's evaluate() recomputed on the host from the same point,
  at the point the solve returned and at disturbed points where every term is active;
* the point the solve returned against the residual block the solve itself reported;
* an out-of-range row index turns every output into NaN (the kernel checks each index, so
  nothing is read out of bounds), and too many rows are refused before anything runs.

Device buffers here are made by torch; the entry point itself allocates nothing. This file is
collected last so that a failure here never hides another test's result.
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle
from sih26_b200 import lpgen
from sih26_b200 import pdhg as P
from tests.test_quality_oracle import edge_lps

pytestmark = pytest.mark.gpu

FIELDS = ("relative_primal", "relative_dual", "relative_gap", "primal_objective",
          "dual_objective", "absolute_primal", "absolute_dual", "gap_as_verified",
          "complementarity")
ORACLE_KEYS = {"relative_primal": "primal", "relative_dual": "dual", "relative_gap": "gap",
               "primal_objective": "primal_objective", "dual_objective": "dual_objective",
               "absolute_primal": "absolute_primal", "absolute_dual": "absolute_dual",
               "gap_as_verified": "gap_as_verified", "complementarity": "complementarity"}


def _lps():
    out = [("uniform_min", lpgen.uniform_planted(2000, 5000, 10, seed=0))]
    out += edge_lps()
    big = lpgen.uniform_planted(300, 750, 6, seed=9)
    big.maximize = True
    out.append(("uniform_max", big))
    out.append(("block_angular", lpgen.block_angular_planted(blocks=4, block_rows=60,
                                                             block_cols=150, nnz_per_col=4,
                                                             linking_rows=8, seed=4)))
    return out


def _lib():
    lib = P.load_library()
    lib.sankhya_pdhg_gpu_residuals_noalloc.argtypes = [C.POINTER(P._Problem), C.c_void_p,
                                                       C.c_void_p, C.c_void_p, C.c_void_p]
    return lib


def _device_problem(lp, torch, keep, row_indices=None):
    dev = "cuda:0"

    def put(a, dtype):
        t = torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)
        keep.append(t)
        return t.data_ptr()

    i32 = C.POINTER(C.c_int32)
    f64 = C.POINTER(C.c_double)
    ri = lp.row_indices if row_indices is None else row_indices
    return P._Problem(
        lp.num_rows, lp.num_cols, lp.num_nonzeros,
        C.cast(put(lp.col_starts, torch.int32), i32), C.cast(put(ri, torch.int32), i32),
        C.cast(put(lp.values, torch.float64), f64), C.cast(put(lp.cost, torch.float64), f64),
        C.cast(put(lp.col_lower, torch.float64), f64), C.cast(put(lp.col_upper, torch.float64), f64),
        C.cast(put(lp.row_lower, torch.float64), f64), C.cast(put(lp.row_upper, torch.float64), f64),
        1 if lp.maximize else 0, float(lp.objective_offset))


def _call(lib, torch, prob, x, rd, stream):
    """One call on `stream`; returns the nine fields as a dict."""
    xd = torch.as_tensor(np.ascontiguousarray(x), dtype=torch.float64, device="cuda:0")
    rdd = torch.as_tensor(np.ascontiguousarray(rd), dtype=torch.float64, device="cuda:0")
    out = torch.full((9,), 12345.0, dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    rc = lib.sankhya_pdhg_gpu_residuals_noalloc(C.byref(prob), xd.data_ptr(), rdd.data_ptr(),
                                                out.data_ptr(), stream.cuda_stream)
    assert rc == 0, lib.sankhya_pdhg_gpu_last_error().decode()
    stream.synchronize()
    return dict(zip(FIELDS, out.cpu().numpy().tolist()))


def _close(got, want, rel, floor):
    # equal values (infinite complementarity of a free column included) agree exactly
    return got == want or abs(got - want) <= rel * abs(want) + floor


@pytest.mark.parametrize("name,lp", _lps(), ids=[n for n, _ in _lps()])
def test_noalloc_matches_the_oracle_and_the_solve_twice_in_a_row(name, lp):
    torch = pytest.importorskip("torch")
    lib = _lib()
    sol = P.solve_pdhg(lp, P.Options(pdhg_tolerance=1e-6, iteration_limit=200000))
    sense = -1.0 if lp.maximize else 1.0
    keep = []
    prob = _device_problem(lp, torch, keep)
    stream = torch.cuda.Stream()
    rng = np.random.default_rng(11)
    points = [("answer", sol.col_value, sol.row_dual)]
    for scale in (1e-3, 0.3):
        points.append((f"disturbed {scale:g}",
                       sol.col_value + scale * rng.standard_normal(lp.num_cols),
                       sol.row_dual + scale * rng.standard_normal(lp.num_rows)))
    for label, x, rd in points:
        want = oracle.oracle_evaluate(lp, x, -sense * rd)  # PDHG sign: y = -sense * row_dual
        for call in range(2):
            got = _call(lib, torch, prob, x, rd, stream)
            for k in FIELDS:
                w = want[ORACLE_KEYS[k]]
                # A x is summed in a different order (atomics), so a residual that is itself
                # at rounding level keeps only an absolute agreement
                floor = 1e-11 if label == "answer" else 1e-13
                assert _close(got[k], w, 1e-12, floor), (name, label, call, k, got[k], w)
        if label == "answer" and sol.status in ("optimal", "feasible"):
            for k in FIELDS:
                assert _close(got[k], sol.residuals[k], 1e-6, 1e-9), (name, k, got[k],
                                                                      sol.residuals[k])


def test_noalloc_flags_a_bad_row_index_and_refuses_oversized_problems():
    torch = pytest.importorskip("torch")
    lib = _lib()
    lp = lpgen.uniform_planted(60, 150, 4, seed=2)
    keep = []
    bad_rows = np.array(lp.row_indices, dtype=np.int32)
    bad_rows[len(bad_rows) // 2] = lp.num_rows  # one index past the last row
    prob = _device_problem(lp, torch, keep, row_indices=bad_rows)
    stream = torch.cuda.Stream()
    x = np.ones(lp.num_cols)
    rd = np.zeros(lp.num_rows)
    for _ in range(2):
        got = _call(lib, torch, prob, x, rd, stream)
        assert all(math.isnan(v) for v in got.values()), got
    # the next call with good indices is right again (the error word is cleared per call)
    good = _device_problem(lp, torch, keep)
    got = _call(lib, torch, good, x, rd, stream)
    want = oracle.oracle_evaluate(lp, x, -rd)
    assert _close(got["absolute_primal"], want["absolute_primal"], 1e-12, 1e-13)

    # more rows than the fixed scratch holds: refused up front, nothing launched
    bad = P._Problem(P.NOALLOC_MAX_ROWS + 1, 1, 0, good.col_starts, good.row_indices,
                     good.values, good.cost, good.col_lower, good.col_upper, good.row_lower,
                     good.row_upper, 0, 0.0)
    out = torch.zeros(9, dtype=torch.float64, device="cuda:0")
    xd = torch.ones(1, dtype=torch.float64, device="cuda:0")
    rc = lib.sankhya_pdhg_gpu_residuals_noalloc(C.byref(bad), xd.data_ptr(), xd.data_ptr(),
                                                out.data_ptr(), None)
    assert rc == 10
    assert "exceed" in lib.sankhya_pdhg_gpu_last_error().decode()
