"""ctypes bindings for the two oracle libraries (see oracle/__init__.py). Test infrastructure."""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle_pdhg.so")
REF_SO = os.path.join(HERE, "_ref", "libsankhya_ref.so")

# sankhya::SolveStatus numeric values -> to_string names (include/sankhya/model.hpp:62-80,
# src/core/model.cpp:19-34)
STATUS_NAMES = {0: "not_solved", 1: "optimal", 2: "infeasible", 3: "unbounded",
                4: "infeasible_or_unbounded", 5: "feasible", 6: "iteration_limit",
                7: "time_limit", 8: "node_limit", 9: "numerical_error", 10: "model_error"}

_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)


class _LP(C.Structure):
    # identical layout for oracle_lp (pdhg_oracle.h) and ref_lp (ref_harness.cpp)
    _fields_ = [("num_rows", C.c_int32), ("num_cols", C.c_int32), ("num_nonzeros", C.c_int32),
                ("col_starts", _i32p), ("row_indices", _i32p), ("values", _f64p),
                ("cost", _f64p), ("col_lower", _f64p), ("col_upper", _f64p),
                ("row_lower", _f64p), ("row_upper", _f64p), ("maximize", C.c_int32),
                ("objective_offset", C.c_double)]


class _Residuals(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "primal", "dual", "gap", "primal_objective", "dual_objective", "absolute_primal",
        "absolute_dual", "gap_as_verified", "complementarity")]


class _OracleOut(C.Structure):
    _fields_ = [("status", C.c_int32), ("converged", C.c_int32), ("iterations", C.c_int64),
                ("attempts", C.c_int64), ("restarts", C.c_int64), ("evaluations", C.c_int64),
                ("spectral_norm", C.c_double), ("final_eta", C.c_double),
                ("final_omega", C.c_double), ("objective", C.c_double),
                ("dual_bound", C.c_double), ("final_residuals", _Residuals)]


class _RefOut(C.Structure):
    _fields_ = [("status", C.c_int32), ("iterations", C.c_int64), ("objective", C.c_double),
                ("dual_bound", C.c_double), ("solve_seconds", C.c_double),
                ("primal_infeasibility", C.c_double), ("dual_infeasibility", C.c_double),
                ("algorithm", C.c_char * 32), ("message", C.c_char * 1024)]


class _PolishOut(C.Structure):
    _fields_ = [("status", C.c_int32), ("polished", C.c_int32), ("iterations", C.c_int64),
                ("polish_iterations", C.c_int64), ("objective", C.c_double),
                ("primal_infeasibility", C.c_double), ("dual_infeasibility", C.c_double),
                ("algorithm", C.c_char * 64), ("message", C.c_char * 1024)]


def _p(a, t):
    return a.ctypes.data_as(t)


class _Pinned:
    """Keeps contiguous copies alive while a C call holds pointers into them."""

    def __init__(self, lp):
        self.cs = np.ascontiguousarray(lp.col_starts, dtype=np.int32)
        self.ri = np.ascontiguousarray(lp.row_indices, dtype=np.int32)
        self.v = np.ascontiguousarray(lp.values, dtype=np.float64)
        self.c = np.ascontiguousarray(lp.cost, dtype=np.float64)
        self.cl = np.ascontiguousarray(lp.col_lower, dtype=np.float64)
        self.cu = np.ascontiguousarray(lp.col_upper, dtype=np.float64)
        self.rl = np.ascontiguousarray(lp.row_lower, dtype=np.float64)
        self.ru = np.ascontiguousarray(lp.row_upper, dtype=np.float64)
        self.s = _LP(lp.num_rows, lp.num_cols, int(self.cs[-1]), _p(self.cs, _i32p),
                     _p(self.ri, _i32p), _p(self.v, _f64p), _p(self.c, _f64p),
                     _p(self.cl, _f64p), _p(self.cu, _f64p), _p(self.rl, _f64p),
                     _p(self.ru, _f64p), 1 if lp.maximize else 0, float(lp.objective_offset))


_libs = {}


def _build(target):
    subprocess.run(["make", "-C", HERE, target], check=True, stdout=subprocess.DEVNULL)


def _oracle():
    if "oracle" not in _libs:
        if not os.path.exists(ORACLE_SO):
            _build("oracle")
        lib = C.CDLL(ORACLE_SO)
        lib.oracle_pdhg_solve.argtypes = [C.POINTER(_LP), C.c_double, C.c_int64, C.c_int,
                                          C.c_int, C.c_int64, _f64p, _f64p, _f64p,
                                          C.POINTER(_OracleOut)]
        lib.oracle_evaluate.restype = _Residuals
        lib.oracle_evaluate.argtypes = [C.POINTER(_LP), _f64p, _f64p, _f64p, _f64p]
        lib.oracle_spectral_norm.restype = C.c_double
        lib.oracle_spectral_norm.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, _f64p, C.c_int,
                                             C.c_uint32]
        lib.oracle_build_scaling.argtypes = [C.POINTER(_LP), _f64p, C.c_int] + [_f64p] * 8
        lib.oracle_uniform_draws.argtypes = [C.c_uint32, C.c_double, C.c_double, C.c_int64,
                                             _f64p]
        lib.oracle_csc_multiply.argtypes = [C.c_int32, C.c_int32, _i32p, _i32p, _f64p, _f64p,
                                            _f64p]
        lib.oracle_csc_transpose_multiply.argtypes = [C.c_int32, _i32p, _i32p, _f64p, _f64p,
                                                      _f64p]
        lib.oracle_primal_step.argtypes = [C.c_int32, C.c_double] + [_f64p] * 7
        _libs["oracle"] = lib
    return _libs["oracle"]


def oracle_available() -> bool:
    try:
        _oracle()
        return True
    except Exception:
        return False


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _ref():
    if "ref" not in _libs:
        lib = C.CDLL(REF_SO)
        lib.ref_pdhg_solve.argtypes = [C.POINTER(_LP), C.c_double, C.c_int64, C.c_double,
                                       C.c_int, C.c_int, C.c_int64, C.c_int, _f64p, _f64p,
                                       _f64p, C.POINTER(_RefOut)]
        lib.ref_build_scaling.argtypes = [C.POINTER(_LP), _f64p, C.c_int] + [_f64p] * 8
        lib.ref_spectral_norm.restype = C.c_double
        lib.ref_spectral_norm.argtypes = [C.POINTER(_LP), C.c_int, C.c_uint]
        lib.ref_farkas_check.argtypes = [C.POINTER(_LP), _f64p, C.c_char_p, C.c_int]
        lib.ref_ray_check.argtypes = [C.POINTER(_LP), _f64p, C.c_char_p, C.c_int]
        lib.ref_qp_solve.argtypes = [C.POINTER(_LP), _i32p, _i32p, _f64p, C.c_double, C.c_int64,
                                     _f64p, _f64p, _f64p, C.POINTER(_RefOut)]
        lib.ref_read_model.argtypes = [C.c_char_p, C.POINTER(_LP), C.c_char_p, C.c_int]
        lib.ref_recompute_quality.argtypes = [C.POINTER(_LP), _f64p, _f64p, _f64p, C.c_double,
                                              _f64p]
        lib.ref_kkt_instance.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, C.POINTER(_LP),
                                         C.POINTER(C.c_double)]
        lib.ref_validate.argtypes = [C.POINTER(_LP), C.c_char_p, C.c_int]
        lib.ref_polish_ipm.argtypes = [C.POINTER(_LP), _f64p, _f64p, _f64p, C.c_int32, C.c_int64,
                                       C.c_char_p, C.c_double, _f64p, _f64p, _f64p,
                                       C.POINTER(_PolishOut), C.c_char_p]
        _libs["ref"] = lib
    return _libs["ref"]


@dataclasses.dataclass
class OracleResult:
    status: str
    iterations: int
    objective: float
    dual_bound: float
    col_value: np.ndarray
    row_dual: np.ndarray
    col_dual: np.ndarray
    attempts: int = 0
    restarts: int = 0
    evaluations: int = 0
    spectral_norm: float = 0.0
    residuals: Optional[dict] = None
    message: str = ""
    solve_seconds: float = 0.0


def _res_dict(r: _Residuals) -> dict:
    return {k: getattr(r, k) for k, _ in _Residuals._fields_}


def oracle_solve(lp, tolerance=1e-4, iteration_limit=-1, restart=True, stop_at_request=False,
                 random_seed=0) -> OracleResult:
    lib = _oracle()
    pin = _Pinned(lp)
    x = np.zeros(lp.num_cols)
    rd = np.zeros(lp.num_rows)
    cd = np.zeros(lp.num_cols)
    out = _OracleOut()
    lib.oracle_pdhg_solve(C.byref(pin.s), tolerance, iteration_limit, int(restart),
                          int(stop_at_request), random_seed, _p(x, _f64p), _p(rd, _f64p),
                          _p(cd, _f64p), C.byref(out))
    return OracleResult(STATUS_NAMES[out.status], out.iterations, out.objective,
                        out.dual_bound, x, rd, cd, out.attempts, out.restarts,
                        out.evaluations, out.spectral_norm, _res_dict(out.final_residuals))


def oracle_evaluate(lp, x, y) -> dict:
    """Unscaled residuals of (x, y), y in PDHG sign (y = -sense * row_dual)."""
    lib = _oracle()
    pin = _Pinned(lp)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    return _res_dict(lib.oracle_evaluate(C.byref(pin.s), _p(x, _f64p), _p(y, _f64p), None,
                                         None))


def oracle_spectral_norm(lp, iterations=30, seed=1) -> float:
    lib = _oracle()
    pin = _Pinned(lp)
    return lib.oracle_spectral_norm(lp.num_rows, lp.num_cols, _p(pin.cs, _i32p),
                                    _p(pin.ri, _i32p), _p(pin.v, _f64p), iterations, seed)


def oracle_uniform_draws(seed, lo, hi, count) -> np.ndarray:
    out = np.zeros(count)
    _oracle().oracle_uniform_draws(seed, lo, hi, count, _p(out, _f64p))
    return out


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def oracle_csc_multiply(num_rows, col_starts, row_indices, values, x) -> np.ndarray:
    """y = A x over a CSC matrix, as the oracle's solve computes it (src/la/sparse.cpp:202-212)."""
    cs = np.ascontiguousarray(col_starts, dtype=np.int32)
    ri = np.ascontiguousarray(row_indices, dtype=np.int32)
    v, xv = _f64(values), _f64(x)
    y = np.zeros(num_rows)
    _oracle().oracle_csc_multiply(num_rows, len(cs) - 1, _p(cs, _i32p), _p(ri, _i32p),
                                  _p(v, _f64p), _p(xv, _f64p), _p(y, _f64p))
    return y


def oracle_csc_transpose_multiply(col_starts, row_indices, values, x) -> np.ndarray:
    """y = A' x over a CSC matrix (per-column gather, src/la/sparse.cpp:214-229)."""
    cs = np.ascontiguousarray(col_starts, dtype=np.int32)
    ri = np.ascontiguousarray(row_indices, dtype=np.int32)
    v, xv = _f64(values), _f64(x)
    y = np.zeros(len(cs) - 1)
    _oracle().oracle_csc_transpose_multiply(len(cs) - 1, _p(cs, _i32p), _p(ri, _i32p),
                                            _p(v, _f64p), _p(xv, _f64p), _p(y, _f64p))
    return y


def oracle_primal_step(tau, x, cost, at_y, lower, upper):
    """The primal step of src/pdhg/pdhg.cpp:393-400: (x', 2x' - x)."""
    x, cost, at_y, lower, upper = (_f64(a) for a in (x, cost, at_y, lower, upper))
    n = len(x)
    x_next, extrapolated = np.zeros(n), np.zeros(n)
    _oracle().oracle_primal_step(n, tau, *(_p(a, _f64p) for a in (x, cost, at_y, lower, upper,
                                                                    x_next, extrapolated)))
    return x_next, extrapolated


def _scaling(fn, lp, min_cost, ruiz):
    pin = _Pinned(lp)
    mc = np.ascontiguousarray(min_cost, dtype=np.float64)
    outs = [np.zeros(lp.num_rows), np.zeros(lp.num_cols), np.zeros(lp.num_nonzeros),
            np.zeros(lp.num_cols), np.zeros(lp.num_cols), np.zeros(lp.num_cols),
            np.zeros(lp.num_rows), np.zeros(lp.num_rows)]
    fn(C.byref(pin.s), _p(mc, _f64p), ruiz, *[_p(o, _f64p) for o in outs])
    keys = ("row_scale", "col_scale", "values", "cost", "col_lower", "col_upper",
            "row_lower", "row_upper")
    return dict(zip(keys, outs))


def oracle_scaling(lp, min_cost, ruiz=10) -> dict:
    return _scaling(_oracle().oracle_build_scaling, lp, min_cost, ruiz)


def ref_scaling(lp, min_cost, ruiz=10) -> dict:
    return _scaling(_ref().ref_build_scaling, lp, min_cost, ruiz)


def ref_spectral_norm(lp, iterations=30, seed=1) -> float:
    pin = _Pinned(lp)
    return _ref().ref_spectral_norm(C.byref(pin.s), iterations, seed)


def ref_solve(lp, tolerance=1e-4, iteration_limit=-1, time_limit=float("inf"), restart=True,
              stop_at_request=False, random_seed=0, log_level=0) -> OracleResult:
    lib = _ref()
    pin = _Pinned(lp)
    x = np.zeros(lp.num_cols)
    rd = np.zeros(lp.num_rows)
    cd = np.zeros(lp.num_cols)
    out = _RefOut()
    rc = lib.ref_pdhg_solve(C.byref(pin.s), tolerance, iteration_limit, time_limit,
                            int(restart), int(stop_at_request), random_seed, log_level,
                            _p(x, _f64p), _p(rd, _f64p), _p(cd, _f64p), C.byref(out))
    if rc != 0:
        raise RuntimeError(out.message.decode())
    return OracleResult(STATUS_NAMES[out.status], out.iterations, out.objective,
                        out.dual_bound, x, rd, cd, message=out.message.decode(),
                        solve_seconds=out.solve_seconds)


def ref_validate(lp) -> str:
    """The reference's Model::validate text for the LP ("" when it passes)."""
    lib = _ref()
    pin = _Pinned(lp)
    why = C.create_string_buffer(512)
    lib.ref_validate(C.byref(pin.s), why, len(why))
    return why.value.decode()


def ref_farkas_check(lp, y) -> tuple[bool, str]:
    pin = _Pinned(lp)
    y = np.ascontiguousarray(y, dtype=np.float64)
    why = C.create_string_buffer(512)
    rc = _ref().ref_farkas_check(C.byref(pin.s), _p(y, _f64p), why, 512)
    return rc == 1, why.value.decode()


def ref_ray_check(lp, d) -> tuple[bool, str]:
    """ray_proves_unbounded (src/core/certificate.cpp:121-218) of the reference build."""
    pin = _Pinned(lp)
    d = np.ascontiguousarray(d, dtype=np.float64)
    why = C.create_string_buffer(512)
    rc = _ref().ref_ray_check(C.byref(pin.s), _p(d, _f64p), why, 512)
    return rc == 1, why.value.decode()


def ref_qp_solve(lp, tolerance=1e-8, iteration_limit=-1) -> OracleResult:
    """qp::solve_convex_qp (src/qp/qp_condat_vu.cpp:150) of the reference build on an LP with
    a Hessian (lp.hessian_*: lower triangle, CSC)."""
    lib = _ref()
    pin = _Pinned(lp)
    hcs = np.ascontiguousarray(lp.hessian_col_starts, dtype=np.int32)
    hri = np.ascontiguousarray(lp.hessian_row_indices, dtype=np.int32)
    hv = np.ascontiguousarray(lp.hessian_values, dtype=np.float64)
    x = np.zeros(lp.num_cols)
    rd = np.zeros(lp.num_rows)
    cd = np.zeros(lp.num_cols)
    out = _RefOut()
    rc = lib.ref_qp_solve(C.byref(pin.s), _p(hcs, _i32p), _p(hri, _i32p), _p(hv, _f64p),
                          tolerance, iteration_limit, _p(x, _f64p), _p(rd, _f64p), _p(cd, _f64p),
                          C.byref(out))
    if rc != 0:
        raise RuntimeError(out.message.decode())
    return OracleResult(STATUS_NAMES[out.status], out.iterations, out.objective,
                        out.dual_bound, x, rd, cd, message=out.message.decode(),
                        solve_seconds=out.solve_seconds)


def ref_read_model(path):
    """Reads an MPS/LP file with the reference reader into an lpgen.LP."""
    from sih26_b200.lpgen import LP

    lib = _ref()
    head = _LP()
    why = C.create_string_buffer(512)
    if lib.ref_read_model(path.encode(), C.byref(head), why, 512) != 0:
        raise RuntimeError(why.value.decode())
    m, n, nnz = head.num_rows, head.num_cols, head.num_nonzeros
    arrs = dict(cs=np.zeros(n + 1, np.int32), ri=np.zeros(nnz, np.int32), v=np.zeros(nnz),
                c=np.zeros(n), cl=np.zeros(n), cu=np.zeros(n), rl=np.zeros(m), ru=np.zeros(m))
    full = _LP(m, n, nnz, _p(arrs["cs"], _i32p), _p(arrs["ri"], _i32p), _p(arrs["v"], _f64p),
               _p(arrs["c"], _f64p), _p(arrs["cl"], _f64p), _p(arrs["cu"], _f64p),
               _p(arrs["rl"], _f64p), _p(arrs["ru"], _f64p), 0, 0.0)
    if lib.ref_read_model(path.encode(), C.byref(full), why, 512) != 0:
        raise RuntimeError(why.value.decode())
    return LP(num_rows=m, num_cols=n, col_starts=arrs["cs"], row_indices=arrs["ri"],
              values=arrs["v"], cost=arrs["c"], col_lower=arrs["cl"], col_upper=arrs["cu"],
              row_lower=arrs["rl"], row_upper=arrs["ru"], maximize=bool(head.maximize),
              objective_offset=head.objective_offset,
              name=os.path.splitext(os.path.basename(path))[0])


STATUS_VALUES = {v: k for k, v in STATUS_NAMES.items()}


def ref_polish_ipm(lp, col_value, row_dual, col_dual, status, iterations, algorithm,
                   scaled_worst, message="") -> dict:
    """The reference's interior-point polish of a first-order answer (ipm::solve_ipm with a
    WarmStart, inside the steps of polish_with_the_interior_point, src/core/solve.cpp:184-243):
    returns the merged answer's status, algorithm, iterations, objective, message (the first
    answer's `message` with the polish's note appended) and point."""
    lib = _ref()
    pin = _Pinned(lp)
    x = np.ascontiguousarray(col_value, dtype=np.float64)
    rd = np.ascontiguousarray(row_dual, dtype=np.float64)
    cd = np.ascontiguousarray(col_dual, dtype=np.float64)
    xo, rdo, cdo = np.zeros(lp.num_cols), np.zeros(lp.num_rows), np.zeros(lp.num_cols)
    out = _PolishOut()
    rc = lib.ref_polish_ipm(C.byref(pin.s), _p(x, _f64p), _p(rd, _f64p), _p(cd, _f64p),
                            STATUS_VALUES[status], int(iterations), algorithm.encode(),
                            float(scaled_worst), _p(xo, _f64p), _p(rdo, _f64p), _p(cdo, _f64p),
                            C.byref(out), message.encode())
    if rc != 0:
        raise RuntimeError(out.message.decode())
    return {"status": STATUS_NAMES[out.status], "polished": bool(out.polished),
            "iterations": out.iterations, "polish_iterations": out.polish_iterations,
            "objective": out.objective, "primal_infeasibility": out.primal_infeasibility,
            "dual_infeasibility": out.dual_infeasibility,
            "algorithm": out.algorithm.decode(), "message": out.message.decode(),
            "col_value": xo, "row_dual": rdo, "col_dual": cdo}


def ref_kkt_instance(seed, max_rows, max_cols, index):
    """Instance `index` of the reference's kkt_lp sequence from mt19937_64(seed)
    (tests/oracles/lp_generator.cpp:122-189, converted by oracle::to_model), as an lpgen.LP,
    with its analytic optimal objective in .optimal_objective."""
    from sih26_b200.lpgen import LP

    lib = _ref()
    head = _LP()
    opt = C.c_double()
    if lib.ref_kkt_instance(seed, max_rows, max_cols, index, C.byref(head), C.byref(opt)) != 0:
        raise RuntimeError("ref_kkt_instance failed")
    m, n, nnz = head.num_rows, head.num_cols, head.num_nonzeros
    arrs = dict(cs=np.zeros(n + 1, np.int32), ri=np.zeros(nnz, np.int32), v=np.zeros(nnz),
                c=np.zeros(n), cl=np.zeros(n), cu=np.zeros(n), rl=np.zeros(m), ru=np.zeros(m))
    full = _LP(m, n, nnz, _p(arrs["cs"], _i32p), _p(arrs["ri"], _i32p), _p(arrs["v"], _f64p),
               _p(arrs["c"], _f64p), _p(arrs["cl"], _f64p), _p(arrs["cu"], _f64p),
               _p(arrs["rl"], _f64p), _p(arrs["ru"], _f64p), 0, 0.0)
    if lib.ref_kkt_instance(seed, max_rows, max_cols, index, C.byref(full), C.byref(opt)) != 0:
        raise RuntimeError("ref_kkt_instance failed")
    return LP(num_rows=m, num_cols=n, col_starts=arrs["cs"], row_indices=arrs["ri"],
              values=arrs["v"], cost=arrs["c"], col_lower=arrs["cl"], col_upper=arrs["cu"],
              row_lower=arrs["rl"], row_upper=arrs["ru"], maximize=bool(head.maximize),
              objective_offset=head.objective_offset, name=f"kkt{index}",
              optimal_objective=float(opt.value))


QUALITY_KEYS = ("primal_infeasibility", "primal_infeasibility_scaled", "dual_infeasibility",
                "dual_infeasibility_scaled", "complementarity_violation", "objective",
                "absolute_gap", "relative_gap")


def ref_recompute_quality(lp, x, row_dual, col_dual, dual_bound) -> dict:
    """Solution::recompute_quality (src/core/model.cpp:228-424) of the reference build."""
    pin = _Pinned(lp)
    arrs = [np.ascontiguousarray(v, dtype=np.float64) for v in (x, row_dual, col_dual)]
    out = np.zeros(8)
    rc = _ref().ref_recompute_quality(C.byref(pin.s), *[_p(a, _f64p) for a in arrs],
                                      float(dual_bound), _p(out, _f64p))
    if rc != 0:
        raise RuntimeError("recompute_quality failed")
    return dict(zip(QUALITY_KEYS, out.tolist()))
