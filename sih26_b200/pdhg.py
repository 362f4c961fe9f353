"""Python face of the GPU PDHG engine, shaped like the reference's own interface.

The reference exposes the path as ``Solution sankhya::pdhg::solve_pdhg(const Model&, const
Options&, Logger&)`` (include/sankhya/pdhg.hpp:15) reading the option rows ``pdhg_tolerance``,
``iteration_limit``, ``time_limit``, ``pdhg_restart``, ``pdhg_stop_at_request`` and
``random_seed`` (src/pdhg/pdhg.cpp:305-315, src/util/options.cpp:83-418). ``solve_pdhg`` here
takes the same options by the same names and returns a ``Solution`` with the reference's
fields and sign conventions, computed by the CUDA library through its C ABI
(include/sankhya_pdhg_gpu.h). There is no CPU fallback: without the library or a GPU the call
raises ``GpuError``.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import math
import os
from typing import List, Optional

import numpy as np

from .lpgen import LP

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "_lib", "libsankhya_pdhg_gpu.so")

# sankhya_pdhg_gpu_status (mirrors sankhya::gpu::GpuStatus, include/sankhya/gpu_runtime.hpp:19-30)
GPU_STATUS = {0: "success", 1: "cuda unavailable", 2: "no compatible cuda device",
              3: "initialization failed", 4: "out of device memory", 5: "kernel launch failed",
              6: "memory copy failed", 7: "device synchronization failed",
              8: "invalid device state", 9: "non-finite numerical output detected",
              10: "invalid argument", 11: "device wait timed out"}

# sankhya_solve_status values (include/sankhya/sankhya.h:53-66) -> SolveStatus names
# (src/core/model.cpp:19-34)
SOLVE_STATUS = {0: "not_solved", 1: "optimal", 2: "feasible", 3: "infeasible", 4: "unbounded",
                5: "iteration_limit", 6: "time_limit", 7: "node_limit", 8: "numerical_error",
                9: "model_error", 10: "infeasible_or_unbounded"}

PRECISIONS = {"fp64": 0, "mixed": 1}
ALGORITHMS = {"reference": 0, "halpern": 1}
PREPS = {"auto": 0, "host": 1, "device": 2}
STOP_RULES = {"reference": 0, "relative_kkt": 1}


class GpuError(RuntimeError):
    """The GPU path could not run; carries the library's status code."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{GPU_STATUS.get(code, code)}: {message}")
        self.code = code


_i32p = C.POINTER(C.c_int32)
_f64p = C.POINTER(C.c_double)


class _Problem(C.Structure):
    _fields_ = [("num_rows", C.c_int32), ("num_cols", C.c_int32), ("num_nonzeros", C.c_int32),
                ("col_starts", _i32p), ("row_indices", _i32p), ("values", _f64p),
                ("cost", _f64p), ("col_lower", _f64p), ("col_upper", _f64p),
                ("row_lower", _f64p), ("row_upper", _f64p), ("maximize", C.c_int32),
                ("objective_offset", C.c_double)]


class _Params(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("iteration_limit", C.c_int64),
                ("time_limit", C.c_double), ("restart", C.c_int32),
                ("stop_at_request", C.c_int32), ("random_seed", C.c_int64),
                ("precision", C.c_int32), ("stop_rule", C.c_int32), ("device", C.c_int32),
                ("verbose", C.c_int32), ("detect_infeasibility", C.c_int32),
                ("mixed_switch_tolerance", C.c_double), ("group_size_rows", C.c_int32),
                ("group_size_cols", C.c_int32), ("grid_blocks", C.c_int32),
                ("profile_kernels", C.c_int32), ("mixed_stall_checks", C.c_int32),
                ("algorithm", C.c_int32), ("autotune", C.c_int32), ("prep", C.c_int32),
                ("qp_assume_convex", C.c_int32), ("reserved", C.c_int32 * 1)]


class _Residuals(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "relative_primal", "relative_dual", "relative_gap", "primal_objective",
        "dual_objective", "absolute_primal", "absolute_dual", "gap_as_verified",
        "complementarity")]


class _Quality(C.Structure):
    _fields_ = [(k, C.c_double) for k in (
        "primal_infeasibility", "primal_infeasibility_scaled", "dual_infeasibility",
        "dual_infeasibility_scaled", "complementarity_violation", "absolute_gap",
        "relative_gap")]


class _Result(C.Structure):
    _fields_ = [("col_value", _f64p), ("row_dual", _f64p), ("col_dual", _f64p),
                ("farkas_dual", _f64p), ("primal_ray", _f64p), ("status", C.c_int32),
                ("converged", C.c_int32), ("iterations", C.c_int64), ("attempts", C.c_int64),
                ("restarts", C.c_int64), ("evaluations", C.c_int64),
                ("fp32_iterations", C.c_int64), ("objective", C.c_double),
                ("dual_bound", C.c_double), ("spectral_norm", C.c_double),
                ("setup_seconds", C.c_double), ("solve_seconds", C.c_double),
                ("total_seconds", C.c_double), ("h2d_bytes", C.c_int64),
                ("d2h_bytes", C.c_int64), ("iterate_kernel_seconds", C.c_double),
                ("iterate_launches", C.c_int64), ("kernel_launches", C.c_int64),
                ("residuals", _Residuals), ("autotuned", C.c_int32),
                ("schedule", C.c_int32 * 4), ("primal_infeasibility", C.c_double),
                ("quality", _Quality), ("message", C.c_char * 512)]


# Every symbol include/sankhya_pdhg_gpu.h declares.
EXPORTED_SYMBOLS = ("sankhya_pdhg_gpu_default_params", "sankhya_pdhg_gpu_solve",
                    "sankhya_pdhg_gpu_last_error", "sankhya_pdhg_gpu_device_count",
                    "sankhya_pdhg_gpu_device_name", "sankhya_pdhg_gpu_residuals_noalloc",
                    "sankhya_pdhg_server_default_config", "sankhya_pdhg_server_create",
                    "sankhya_pdhg_server_submit", "sankhya_pdhg_server_step",
                    "sankhya_pdhg_server_result", "sankhya_pdhg_server_free",
                    "sankhya_pdhg_server_get_stats",
                    "sankhya_pdhg_gpu_batch_solve", "sankhya_pdhg_wire_size",
                    "sankhya_pdhg_wire_write", "sankhya_pdhg_wire_view",
                    "sankhya_qp_gpu_solve")

# SANKHYA_PDHG_NOALLOC_MAX_ROWS: rows the allocation-free residual check's fixed scratch holds
NOALLOC_MAX_ROWS = 516064

_lib: Optional[C.CDLL] = None


def load_library() -> C.CDLL:
    """Loads the in-tree CUDA library; raises GpuError when it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise GpuError(1, f"{LIBPATH} is not built (python -m sih26_b200.build)")
        lib = C.CDLL(LIBPATH)
        lib.sankhya_pdhg_gpu_default_params.argtypes = [C.POINTER(_Params)]
        lib.sankhya_pdhg_gpu_solve.argtypes = [C.POINTER(_Problem), C.POINTER(_Params),
                                               C.POINTER(_Result)]
        lib.sankhya_pdhg_gpu_last_error.restype = C.c_char_p
        lib.sankhya_pdhg_gpu_device_name.argtypes = [C.c_int, C.c_char_p, C.c_int]
        _lib = lib
    return _lib


def device_count() -> int:
    return load_library().sankhya_pdhg_gpu_device_count()


class Options:
    """The option rows the PDHG path reads, with the reference's names and defaults
    (src/util/options.cpp:83-418), plus the GPU rows this engine adds."""

    _SPECS = {
        # name: (type, default)
        "pdhg_tolerance": (float, 1e-4),
        "iteration_limit": (int, -1),
        "time_limit": (float, math.inf),
        "pdhg_restart": (bool, True),
        "pdhg_stop_at_request": (bool, False),
        "random_seed": (int, 0),
        "log_to_console": (bool, False),
        "pdhg_precision": (str, "fp64"),
        "pdhg_stop_rule": (str, "reference"),
        "pdhg_mixed_switch_tolerance": (float, 0.0),
        "pdhg_detect_infeasibility": (bool, True),
        "gpu_device": (int, 0),
        "pdhg_lanes_rows": (int, 0),
        "pdhg_lanes_cols": (int, 0),
        "pdhg_grid_blocks": (int, 0),
        "pdhg_profile_kernels": (bool, False),
        "pdhg_mixed_stall_checks": (int, 0),
        "pdhg_algorithm": (str, "reference"),
        "pdhg_autotune": (bool, False),
        "pdhg_prep": (str, "auto"),
        "qp_tolerance": (float, 1e-8),
        "qp_assume_convex": (bool, False),
    }

    def __init__(self, **values):
        self._v = {k: d for k, (_, d) in self._SPECS.items()}
        for k, v in values.items():
            self.set(k, v)

    def set(self, name, value):
        if name not in self._SPECS:
            raise KeyError(f"no such option: {name}")
        typ = self._SPECS[name][0]
        if typ is bool and isinstance(value, str):
            value = value.lower() in ("1", "true", "on", "yes")
        if typ is str:
            allowed = {"pdhg_precision": PRECISIONS, "pdhg_stop_rule": STOP_RULES,
                       "pdhg_algorithm": ALGORITHMS, "pdhg_prep": PREPS}.get(name)
            if allowed is not None and value not in allowed:
                raise ValueError(f"{name} must be one of {sorted(allowed)}")
        self._v[name] = typ(value)

    def set_from_string(self, text: str):
        """`name=value`, the CLI's --option form (src/util/options.cpp:481)."""
        name, _, value = text.partition("=")
        self.set(name.strip(), value.strip())

    def get(self, name):
        return self._v[name]

    get_double = get_int = get_bool = get_string = get
    set_double = set_int = set_bool = set_string = set


@dataclasses.dataclass
class Solution:
    """The reference's Solution fields this path fills (include/sankhya/model.hpp:233-374)."""

    status: str
    objective: float
    dual_bound: float
    col_value: np.ndarray
    row_dual: np.ndarray
    col_dual: np.ndarray
    iterations: int
    solve_seconds: float
    algorithm: str
    message: str
    primal_infeasibility: float = 0.0
    # Solution::recompute_quality's figures of the reported point, measured on the device:
    # primal_infeasibility(_scaled), dual_infeasibility(_scaled), complementarity_violation,
    # absolute_gap, relative_gap (src/core/model.cpp:228-424)
    quality: Optional[dict] = None
    farkas_dual: Optional[np.ndarray] = None
    primal_ray: Optional[np.ndarray] = None
    # engine detail
    attempts: int = 0
    restarts: int = 0
    evaluations: int = 0
    fp32_iterations: int = 0
    spectral_norm: float = 0.0
    residuals: Optional[dict] = None
    setup_seconds: float = 0.0
    device_seconds: float = 0.0
    h2d_bytes: int = 0
    d2h_bytes: int = 0
    iterate_kernel_seconds: float = 0.0
    iterate_launches: int = 0
    kernel_launches: int = 0
    autotuned: int = 0
    schedule: tuple = ()

    def has_primal_values(self) -> bool:
        return self.status in ("optimal", "feasible")


def _arr(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def primal_infeasibility_host(lp: LP, x: np.ndarray) -> float:
    """Max row/column bound violation (Solution::recompute_quality, src/core/model.cpp:228-283),
    on the host; the solves report the same figure computed on the device."""
    act = lp.to_scipy_csc() @ x if lp.num_rows else np.zeros(0)
    fin = lambda v: np.abs(v) < 1e30  # noqa: E731
    viol = [0.0]
    for lo, val in ((lp.col_lower, x), (lp.row_lower, act)):
        m = fin(lo)
        if m.any():
            viol.append(float(np.max(lo[m] - val[m])))
    for hi, val in ((lp.col_upper, x), (lp.row_upper, act)):
        m = fin(hi)
        if m.any():
            viol.append(float(np.max(val[m] - hi[m])))
    return max(0.0, max(viol))


def solve_pdhg(model: LP, options: Optional[Options] = None) -> Solution:
    """GPU successor of sankhya::pdhg::solve_pdhg (src/pdhg/pdhg.cpp:267-726)."""
    opt = options or Options()
    lib = load_library()
    cs = _arr(model.col_starts, np.int32)
    ri = _arr(model.row_indices, np.int32)
    vals = _arr(model.values, np.float64)
    vecs = [_arr(v, np.float64) for v in (model.cost, model.col_lower, model.col_upper,
                                           model.row_lower, model.row_upper)]
    prob = _Problem(model.num_rows, model.num_cols, int(cs[-1]) if cs.size else 0,
                    cs.ctypes.data_as(_i32p), ri.ctypes.data_as(_i32p),
                    vals.ctypes.data_as(_f64p), *[v.ctypes.data_as(_f64p) for v in vecs],
                    1 if model.maximize else 0, float(model.objective_offset))
    prm = _params(opt, lib)
    n, m = model.num_cols, model.num_rows
    x = np.zeros(n)
    rd = np.zeros(m)
    cd = np.zeros(n)
    fk = np.zeros(m)
    ray = np.zeros(n)
    res = _Result()
    res.col_value = x.ctypes.data_as(_f64p)
    res.row_dual = rd.ctypes.data_as(_f64p)
    res.col_dual = cd.ctypes.data_as(_f64p)
    res.farkas_dual = fk.ctypes.data_as(_f64p)
    res.primal_ray = ray.ctypes.data_as(_f64p)
    code = lib.sankhya_pdhg_gpu_solve(C.byref(prob), C.byref(prm), C.byref(res))
    if code != 0:
        raise GpuError(code, lib.sankhya_pdhg_gpu_last_error().decode())
    status = SOLVE_STATUS[res.status]
    r = res.residuals
    sol = Solution(
        status=status, objective=res.objective, dual_bound=res.dual_bound, col_value=x,
        row_dual=rd, col_dual=cd, iterations=res.iterations,
        solve_seconds=res.total_seconds, algorithm="pdhg-gpu",
        message=res.message.decode(errors="replace"),
        farkas_dual=fk if status == "infeasible" else None,
        primal_ray=ray if status in ("unbounded", "infeasible_or_unbounded") else None,
        attempts=res.attempts, restarts=res.restarts, evaluations=res.evaluations,
        fp32_iterations=res.fp32_iterations, spectral_norm=res.spectral_norm,
        residuals={k: getattr(r, k) for k, _ in _Residuals._fields_},
        setup_seconds=res.setup_seconds, device_seconds=res.solve_seconds,
        h2d_bytes=res.h2d_bytes, d2h_bytes=res.d2h_bytes,
        iterate_kernel_seconds=res.iterate_kernel_seconds, iterate_launches=res.iterate_launches,
        kernel_launches=res.kernel_launches, autotuned=res.autotuned,
        schedule=tuple(res.schedule))
    if status not in ("model_error", "infeasible"):
        # computed on the device; for UNBOUNDED, of the feasible point the ray starts from
        sol.primal_infeasibility = res.primal_infeasibility
        sol.quality = _quality(res)
    return sol


def _quality(res) -> dict:
    return {k: getattr(res.quality, k) for k, _ in _Quality._fields_}


# ---- convex QP (sankhya_qp_gpu_solve) --------------------------------------------------------

class _Hessian(C.Structure):
    _fields_ = [("num_nonzeros", C.c_int32), ("col_starts", _i32p), ("row_indices", _i32p),
                ("values", _f64p)]


def solve_qp(model: LP, options: Optional[Options] = None) -> Solution:
    """GPU successor of qp::solve_convex_qp (src/qp/qp_condat_vu.cpp:150): `model` carries Q's
    lower triangle in hessian_col_starts / hessian_row_indices / hessian_values; the options
    read are qp_tolerance, iteration_limit, time_limit, gpu_device and qp_assume_convex."""
    opt = options or Options()
    lib = load_library()
    if not getattr(lib, "_qp_bound", False):
        lib.sankhya_qp_gpu_solve.argtypes = [C.POINTER(_Problem), C.POINTER(_Hessian),
                                             C.POINTER(_Params), C.POINTER(_Result)]
        lib._qp_bound = True
    held = _Held(model)
    n = model.num_cols
    hcs = _arr(model.hessian_col_starts if model.hessian_col_starts is not None
               else np.zeros(n + 1), np.int32)
    hri = _arr(model.hessian_row_indices if model.hessian_row_indices is not None
               else np.zeros(0), np.int32)
    hv = _arr(model.hessian_values if model.hessian_values is not None else np.zeros(0),
              np.float64)
    hes = _Hessian(int(hcs[-1]) if hcs.size else 0, hcs.ctypes.data_as(_i32p),
                   hri.ctypes.data_as(_i32p), hv.ctypes.data_as(_f64p))
    prm = _params(opt, lib)
    prm.tolerance = opt.get("qp_tolerance")
    prm.qp_assume_convex = int(opt.get("qp_assume_convex"))
    out = _Outputs(model)
    code = lib.sankhya_qp_gpu_solve(C.byref(held.problem), C.byref(hes), C.byref(prm),
                                    C.byref(out.res))
    if code != 0:
        raise GpuError(code, lib.sankhya_pdhg_gpu_last_error().decode())
    sol = out.solution(model)
    sol.algorithm = "qp-condat-vu-gpu"
    return sol


# ---- request wire format (sankhya_pdhg_wire_*) ----------------------------------------------

def _bind_wire(lib):
    if getattr(lib, "_wire_bound", False):
        return
    lib.sankhya_pdhg_wire_size.argtypes = [C.POINTER(_Problem)]
    lib.sankhya_pdhg_wire_size.restype = C.c_size_t
    lib.sankhya_pdhg_wire_write.argtypes = [C.POINTER(_Problem), C.c_void_p, C.c_size_t]
    lib.sankhya_pdhg_wire_view.argtypes = [C.c_void_p, C.c_size_t, C.POINTER(_Problem)]
    lib._wire_bound = True


def to_wire(model: LP) -> np.ndarray:
    """The wire form of an LP (include/sankhya_pdhg_gpu.h): an 8-byte-aligned uint8 array."""
    lib = load_library()
    _bind_wire(lib)
    held = _Held(model)
    size = lib.sankhya_pdhg_wire_size(C.byref(held.problem))
    buf = np.zeros((size + 7) // 8, dtype=np.uint64).view(np.uint8)[:size]
    code = lib.sankhya_pdhg_wire_write(C.byref(held.problem), buf.ctypes.data, size)
    if code != 0:
        raise GpuError(code, lib.sankhya_pdhg_gpu_last_error().decode())
    return buf


def from_wire(buffer) -> LP:
    """An LP read from a wire buffer through sankhya_pdhg_wire_view (the arrays are copied out
    of the buffer, so it need not outlive the result)."""
    lib = load_library()
    _bind_wire(lib)
    raw = np.frombuffer(buffer, dtype=np.uint8)
    if raw.ctypes.data % 8:
        raw = np.frombuffer(raw.tobytes(), dtype=np.uint8)
    aligned = np.zeros((raw.size + 7) // 8, dtype=np.uint64).view(np.uint8)[:raw.size]
    aligned[:] = raw
    prob = _Problem()
    code = lib.sankhya_pdhg_wire_view(aligned.ctypes.data, aligned.size, C.byref(prob))
    if code != 0:
        raise GpuError(code, lib.sankhya_pdhg_gpu_last_error().decode())
    m, n, nnz = prob.num_rows, prob.num_cols, prob.num_nonzeros

    def arr(ptr, count, dtype):
        if count == 0:
            return np.zeros(0, dtype=dtype)
        return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype, copy=True)

    lp = LP(num_rows=m, num_cols=n, col_starts=arr(prob.col_starts, n + 1, np.int32),
            row_indices=arr(prob.row_indices, nnz, np.int32), values=arr(prob.values, nnz, np.float64),
            cost=arr(prob.cost, n, np.float64), col_lower=arr(prob.col_lower, n, np.float64),
            col_upper=arr(prob.col_upper, n, np.float64), row_lower=arr(prob.row_lower, m, np.float64),
            row_upper=arr(prob.row_upper, m, np.float64), maximize=bool(prob.maximize),
            objective_offset=float(prob.objective_offset))
    return lp


class WireRequest:
    """A request held in its wire form: the 8-byte-aligned buffer and the problem struct that
    sankhya_pdhg_wire_view points into it. The solves below read the LP in place; nothing is
    copied out of the buffer on the host."""

    def __init__(self, buffer):
        lib = load_library()
        _bind_wire(lib)
        raw = np.frombuffer(buffer, dtype=np.uint8)
        self.buffer = np.zeros((raw.size + 7) // 8, dtype=np.uint64).view(np.uint8)[:raw.size]
        self.buffer[:] = raw
        self.problem = _Problem()
        code = lib.sankhya_pdhg_wire_view(self.buffer.ctypes.data, self.buffer.size,
                                          C.byref(self.problem))
        if code != 0:
            raise GpuError(code, lib.sankhya_pdhg_gpu_last_error().decode())
        self.num_rows = self.problem.num_rows
        self.num_cols = self.problem.num_cols


def solve_wire(request: WireRequest, options: Optional[Options] = None) -> Solution:
    """sankhya_pdhg_gpu_solve on an LP read in place from its wire buffer."""
    opt = options or Options()
    lib = load_library()
    prm = _params(opt, lib)
    out = _Outputs(request)
    code = lib.sankhya_pdhg_gpu_solve(C.byref(request.problem), C.byref(prm), C.byref(out.res))
    if code != 0:
        raise GpuError(code, lib.sankhya_pdhg_gpu_last_error().decode())
    sol = out.solution(request)
    sol.algorithm = "pdhg-gpu"
    return sol


# ---- many LPs at once (the served / batched engine) ---------------------------------------

class _ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("memory_fraction", C.c_double),
                ("pool_bytes", C.c_int64), ("max_active", C.c_int32),
                ("chunk_attempts", C.c_int64), ("cluster_min_nnz", C.c_int64),
                ("clusters", C.c_int32), ("solo_min_nnz", C.c_int32),
                ("reserved", C.c_int32 * 6)]


class _ServerStats(C.Structure):
    _fields_ = [("chunk_attempts", C.c_int64), ("chunk_source", C.c_int32),
                ("clusters", C.c_int32), ("rounds", C.c_int64), ("last_round_ms", C.c_double),
                ("family", C.c_char * 192), ("reserved", C.c_int32 * 4)]


def _bind_server(lib):
    if getattr(lib, "_server_bound", False):
        return
    lib.sankhya_pdhg_server_default_config.argtypes = [C.POINTER(_ServerConfig)]
    lib.sankhya_pdhg_server_create.argtypes = [C.POINTER(_ServerConfig), C.POINTER(C.c_void_p)]
    lib.sankhya_pdhg_server_submit.argtypes = [C.c_void_p, C.POINTER(_Problem), C.POINTER(_Params),
                                               C.POINTER(C.c_int64)]
    lib.sankhya_pdhg_server_step.argtypes = [C.c_void_p, C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    lib.sankhya_pdhg_server_result.argtypes = [C.c_void_p, C.c_int64, C.POINTER(_Result)]
    lib.sankhya_pdhg_server_free.argtypes = [C.c_void_p]
    lib.sankhya_pdhg_server_get_stats.argtypes = [C.c_void_p, C.POINTER(_ServerStats)]
    lib.sankhya_pdhg_gpu_batch_solve.argtypes = [C.POINTER(_Problem), C.c_int32,
                                                 C.POINTER(_Params), C.POINTER(_Result)]
    lib._server_bound = True


def _params(opt: Options, lib) -> _Params:
    prm = _Params()
    lib.sankhya_pdhg_gpu_default_params(C.byref(prm))
    prm.tolerance = opt.get("pdhg_tolerance")
    prm.iteration_limit = opt.get("iteration_limit")
    prm.time_limit = opt.get("time_limit")
    prm.restart = int(opt.get("pdhg_restart"))
    prm.stop_at_request = int(opt.get("pdhg_stop_at_request"))
    prm.random_seed = opt.get("random_seed")
    prm.precision = PRECISIONS[opt.get("pdhg_precision")]
    prm.stop_rule = STOP_RULES[opt.get("pdhg_stop_rule")]
    prm.device = opt.get("gpu_device")
    prm.verbose = int(opt.get("log_to_console"))
    prm.detect_infeasibility = int(opt.get("pdhg_detect_infeasibility"))
    prm.mixed_switch_tolerance = opt.get("pdhg_mixed_switch_tolerance")
    prm.group_size_rows = opt.get("pdhg_lanes_rows")
    prm.group_size_cols = opt.get("pdhg_lanes_cols")
    prm.grid_blocks = opt.get("pdhg_grid_blocks")
    prm.profile_kernels = int(opt.get("pdhg_profile_kernels"))
    prm.mixed_stall_checks = opt.get("pdhg_mixed_stall_checks")
    prm.algorithm = ALGORITHMS[opt.get("pdhg_algorithm")]
    prm.autotune = int(opt.get("pdhg_autotune"))
    prm.prep = PREPS[opt.get("pdhg_prep")]
    return prm


class _Held:
    """A problem struct and the contiguous arrays it points into."""

    def __init__(self, model: LP):
        self.arrays = [_arr(model.col_starts, np.int32), _arr(model.row_indices, np.int32)] + [
            _arr(v, np.float64) for v in (model.values, model.cost, model.col_lower,
                                          model.col_upper, model.row_lower, model.row_upper)]
        cs, ri, vals, *vecs = self.arrays
        self.problem = _Problem(model.num_rows, model.num_cols, int(cs[-1]) if cs.size else 0,
                                cs.ctypes.data_as(_i32p), ri.ctypes.data_as(_i32p),
                                vals.ctypes.data_as(_f64p),
                                *[v.ctypes.data_as(_f64p) for v in vecs],
                                1 if model.maximize else 0, float(model.objective_offset))


class _Outputs:
    def __init__(self, model: LP):
        n, m = model.num_cols, model.num_rows
        self.x, self.cd, self.rd, self.fk, self.ray = (np.zeros(n), np.zeros(n), np.zeros(m),
                                                       np.zeros(m), np.zeros(n))
        self.res = _Result()
        self.res.col_value = self.x.ctypes.data_as(_f64p)
        self.res.col_dual = self.cd.ctypes.data_as(_f64p)
        self.res.row_dual = self.rd.ctypes.data_as(_f64p)
        self.res.farkas_dual = self.fk.ctypes.data_as(_f64p)
        self.res.primal_ray = self.ray.ctypes.data_as(_f64p)

    def solution(self, model: LP) -> Solution:
        res = self.res
        status = SOLVE_STATUS[res.status]
        r = res.residuals
        sol = Solution(
            status=status, objective=res.objective, dual_bound=res.dual_bound,
            col_value=self.x, row_dual=self.rd, col_dual=self.cd, iterations=res.iterations,
            solve_seconds=res.total_seconds, algorithm="pdhg-gpu-batch",
            message=res.message.decode(errors="replace"),
            farkas_dual=self.fk if status == "infeasible" else None,
            primal_ray=self.ray if status in ("unbounded", "infeasible_or_unbounded") else None,
            attempts=res.attempts, restarts=res.restarts, evaluations=res.evaluations,
            spectral_norm=res.spectral_norm,
            residuals={k: getattr(r, k) for k, _ in _Residuals._fields_},
            setup_seconds=res.setup_seconds, device_seconds=res.solve_seconds,
            kernel_launches=res.kernel_launches)
        if status not in ("model_error", "infeasible"):
            sol.primal_infeasibility = res.primal_infeasibility  # computed on the device
            sol.quality = _quality(res)
        return sol


def batch_solve(models, options: Optional[Options] = None):
    """Solves independent LPs concurrently on one GPU (sankhya_pdhg_gpu_batch_solve)."""
    opt = options or Options()
    lib = load_library()
    _bind_server(lib)
    held = [_Held(m) for m in models]
    outs = [_Outputs(m) for m in models]
    probs = (_Problem * len(models))(*[h.problem for h in held])
    results = (_Result * len(models))(*[o.res for o in outs])
    prm = _params(opt, lib)
    code = lib.sankhya_pdhg_gpu_batch_solve(probs, len(models), C.byref(prm), results)
    if code != 0:
        raise GpuError(code, lib.sankhya_pdhg_gpu_last_error().decode())
    sols = []
    for k, m in enumerate(models):
        outs[k].res = results[k]
        sols.append(outs[k].solution(m))
    return sols


class Server:
    """A resident GPU server for many LPs (sankhya_pdhg_server_*): submit() queues an LP,
    step() admits what fits and runs one launch over every active LP, result() collects.
    LPs with at least `cluster_min_nnz` nonzeros run on an 8-block thread-block cluster
    (`clusters` of them; 0 = chosen every round from the large LPs' share of the active
    nonzeros), the others on one block each; LPs with at least `solo_min_nnz` nonzeros are
    solved one per step on the whole GPU by the single-LP engine. `chunk_attempts` = -1 lets
    the server search the attempts per launch for the most LPs finished per second itself (the
    choice changes when an LP pauses, not its answer); stats() reports the setting."""

    CHUNK_SOURCES = ("configured", "tuned", "cache")

    def __init__(self, device: int = 0, memory_fraction: float = 0.8, pool_bytes: int = 0,
                 max_active: int = 4096, chunk_attempts: int = -1,
                 cluster_min_nnz: int = 16384, clusters: int = 0,
                 solo_min_nnz: int = 0):
        self.lib = load_library()
        _bind_server(self.lib)
        cfg = _ServerConfig()
        self.lib.sankhya_pdhg_server_default_config(C.byref(cfg))
        cfg.device, cfg.memory_fraction, cfg.pool_bytes = device, memory_fraction, pool_bytes
        cfg.max_active, cfg.chunk_attempts = max_active, chunk_attempts
        cfg.cluster_min_nnz, cfg.clusters = cluster_min_nnz, clusters
        cfg.solo_min_nnz = solo_min_nnz
        self.handle = C.c_void_p()
        code = self.lib.sankhya_pdhg_server_create(C.byref(cfg), C.byref(self.handle))
        if code != 0:
            raise GpuError(code, self.lib.sankhya_pdhg_gpu_last_error().decode())
        self.pending = {}

    def submit(self, model: LP, options: Optional[Options] = None) -> int:
        held = _Held(model)
        prm = _params(options or Options(), self.lib)
        ticket = C.c_int64()
        code = self.lib.sankhya_pdhg_server_submit(self.handle, C.byref(held.problem),
                                                   C.byref(prm), C.byref(ticket))
        if code != 0:
            raise GpuError(code, self.lib.sankhya_pdhg_gpu_last_error().decode())
        self.pending[ticket.value] = model
        return ticket.value

    def submit_wire(self, request: WireRequest, options: Optional[Options] = None) -> int:
        """Queues an LP read in place from its wire buffer (the server copies what it keeps)."""
        prm = _params(options or Options(), self.lib)
        ticket = C.c_int64()
        code = self.lib.sankhya_pdhg_server_submit(self.handle, C.byref(request.problem),
                                                   C.byref(prm), C.byref(ticket))
        if code != 0:
            raise GpuError(code, self.lib.sankhya_pdhg_gpu_last_error().decode())
        self.pending[ticket.value] = request
        return ticket.value

    def step(self):
        a, w, f = C.c_int32(), C.c_int32(), C.c_int32()
        code = self.lib.sankhya_pdhg_server_step(self.handle, C.byref(a), C.byref(w), C.byref(f))
        if code != 0:
            raise GpuError(code, self.lib.sankhya_pdhg_gpu_last_error().decode())
        return a.value, w.value, f.value

    def result(self, ticket: int) -> Optional[Solution]:
        model = self.pending[ticket]
        out = _Outputs(model)
        code = self.lib.sankhya_pdhg_server_result(self.handle, ticket, C.byref(out.res))
        if code == 12:
            return None
        if code != 0:
            raise GpuError(code, self.lib.sankhya_pdhg_gpu_last_error().decode())
        del self.pending[ticket]
        return out.solution(model)

    def solve_all(self, models, options: Optional[Options] = None) -> List[Solution]:
        """Submits every model, steps until all have finished, returns the answers in order."""
        tickets = [self.submit(m, options) for m in models]
        done = {}
        while len(done) < len(tickets):
            active, waiting, _ = self.step()
            for t in tickets:
                if t not in done:
                    r = self.result(t)
                    if r is not None:
                        done[t] = r
            if active == 0 and waiting == 0 and len(done) < len(tickets):
                raise GpuError(1, "server idle with unfinished tickets")
        return [done[t] for t in tickets]

    def stats(self) -> dict:
        """The current launch settings: chunk_attempts (0 = each LP to its end), where it
        came from, the clusters of the launch graph, launches so far, the last launch's ms."""
        st = _ServerStats()
        code = self.lib.sankhya_pdhg_server_get_stats(self.handle, C.byref(st))
        if code != 0:
            raise GpuError(code, self.lib.sankhya_pdhg_gpu_last_error().decode())
        return {"chunk_attempts": st.chunk_attempts,
                "chunk_source": self.CHUNK_SOURCES[st.chunk_source],
                "clusters": st.clusters, "rounds": st.rounds, "last_round_ms": st.last_round_ms,
                "family": st.family.decode()}

    def close(self):
        if self.handle:
            self.lib.sankhya_pdhg_server_free(self.handle)
            self.handle = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
