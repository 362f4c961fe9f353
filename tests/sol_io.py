"""MPS and .sol files for answers the GPU returned, so the reference's independent verifier
(tools/verify_solution.py, which reads a model file and a solution file as text) can judge
them.

* ``write_mps``: free-format MPS of an LP (ROWS / COLUMNS / RHS / RANGES / BOUNDS, OBJSENSE
  for maximisation, the objective offset as the negated RHS of the objective row), every
  number written with 17 significant digits so it reads back exactly.
* ``write_sol``: the solution-file layout of the reference's writer (src/io/writer.cpp:
  114-216): a header of ``key value`` lines, then either a ``farkas`` block alone (a verdict
  without a point, ``infeasible``) or the ``columns`` block (value, reduced cost, basis
  status) and the ``rows`` block (activity, dual, basis status), plus a ``ray`` block for
  ``unbounded``. Row and column names are R<i> and C<j>.
"""
from __future__ import annotations

import math

import numpy as np


def _num(v: float) -> str:
    v = float(v)
    if math.isinf(v):
        return "inf" if v > 0 else "-inf"
    return f"{v:.17g}"


def _finite(v: float) -> bool:
    return abs(v) < 1e30


def write_mps(lp, path: str) -> None:
    m, n = lp.num_rows, lp.num_cols
    lines = [f"NAME {lp.name or 'lp'}"]
    if lp.maximize:
        lines += ["OBJSENSE", "    MAX"]
    lines.append("ROWS")
    lines.append(" N OBJ")
    kinds, rhs, rng = [], [], []
    for i in range(m):
        lo, hi = float(lp.row_lower[i]), float(lp.row_upper[i])
        if _finite(lo) and _finite(hi):
            if lo == hi:
                kinds.append("E"); rhs.append(lo); rng.append(None)  # noqa: E702
            else:
                kinds.append("G"); rhs.append(lo); rng.append(hi - lo)  # noqa: E702
        elif _finite(lo):
            kinds.append("G"); rhs.append(lo); rng.append(None)  # noqa: E702
        elif _finite(hi):
            kinds.append("L"); rhs.append(hi); rng.append(None)  # noqa: E702
        else:
            raise ValueError(f"row {i} is free; not representable as a constraint row here")
        lines.append(f" {kinds[-1]} R{i}")
    lines.append("COLUMNS")
    cs, ri, vals = lp.col_starts, lp.row_indices, lp.values
    for j in range(n):
        if lp.cost[j] != 0.0:
            lines.append(f"    C{j} OBJ {_num(lp.cost[j])}")
        for k in range(int(cs[j]), int(cs[j + 1])):
            lines.append(f"    C{j} R{int(ri[k])} {_num(vals[k])}")
        if lp.cost[j] == 0.0 and cs[j] == cs[j + 1]:
            lines.append(f"    C{j} OBJ 0")
    lines.append("RHS")
    for i in range(m):
        if rhs[i] != 0.0:
            lines.append(f"    RHS R{i} {_num(rhs[i])}")
    if lp.objective_offset != 0.0:
        lines.append(f"    RHS OBJ {_num(-lp.objective_offset)}")
    if any(r is not None for r in rng):
        lines.append("RANGES")
        for i in range(m):
            if rng[i] is not None:
                lines.append(f"    RNG R{i} {_num(rng[i])}")
    lines.append("BOUNDS")
    for j in range(n):
        lo, hi = float(lp.col_lower[j]), float(lp.col_upper[j])
        flo, fhi = _finite(lo), _finite(hi)
        if flo and fhi and lo == hi:
            lines.append(f" FX BND C{j} {_num(lo)}")
        elif not flo and not fhi:
            lines.append(f" FR BND C{j}")
        else:
            if not flo:
                lines.append(f" MI BND C{j}")
            elif lo != 0.0 or fhi:
                lines.append(f" LO BND C{j} {_num(lo)}")
            if fhi:
                lines.append(f" UP BND C{j} {_num(hi)}")
    lines.append("ENDATA")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def write_sol(lp, sol, path: str) -> None:
    """`sol`: a pdhg.Solution (or anything with status, objective, dual_bound, col_value,
    row_dual, col_dual, farkas_dual, primal_ray, iterations, primal_infeasibility)."""
    m, n = lp.num_rows, lp.num_cols
    cert = ("farkas" if getattr(sol, "farkas_dual", None) is not None
            else "ray" if getattr(sol, "primal_ray", None) is not None else "none")
    q = getattr(sol, "quality", None) or {}
    head = [
        "# SANKHYA solution file",
        "# generated-by sih26_b200 (GPU PDHG)",
        "# All numbers carry 17 significant digits and round-trip exactly.",
        f"model {lp.name or '(unnamed)'}",
        "source (generated)",
        f"sense {'maximize' if lp.maximize else 'minimize'}",
        f"status {sol.status}",
        f"algorithm {getattr(sol, 'algorithm', 'pdhg-gpu')}",
        f"objective {_num(sol.objective)}",
        f"dual_bound {_num(sol.dual_bound)}",
        "mip_relative_gap 0.0001",
        "mip_absolute_gap 9.9999999999999995e-07",
        f"objective_offset {_num(lp.objective_offset)}",
        f"certificate {cert}",
        f"rows {m}",
        f"columns {n}",
        f"iterations {int(sol.iterations)}",
        "nodes 0",
        f"primal_infeasibility {_num(getattr(sol, 'primal_infeasibility', 0.0))}",
        f"dual_infeasibility {_num(q.get('dual_infeasibility', 0.0))}",
        "integrality_violation 0",
    ]
    body = []
    if sol.status in ("infeasible", "numerical_error", "model_error", "not_solved"):
        if cert == "farkas":
            body.append(f"begin farkas {m}")
            body += [f"R{i} {_num(v)}" for i, v in enumerate(sol.farkas_dual)]
            body.append("end farkas")
    else:
        x = np.asarray(sol.col_value, dtype=np.float64)
        act = lp.to_scipy_csc() @ x if m else np.zeros(0)
        body.append(f"begin columns {n}")
        body += [f"C{j} {_num(x[j])} {_num(sol.col_dual[j])} unknown" for j in range(n)]
        body.append("end columns")
        body.append(f"begin rows {m}")
        body += [f"R{i} {_num(act[i])} {_num(sol.row_dual[i])} unknown" for i in range(m)]
        body.append("end rows")
        if sol.status in ("unbounded", "infeasible_or_unbounded") and cert == "ray":
            body.append(f"begin ray {n}")
            body += [f"C{j} {_num(v)}" for j, v in enumerate(sol.primal_ray)]
            body.append("end ray")
    with open(path, "w") as f:
        f.write("\n".join(head) + "\n\n" + "\n".join(body) + "\n")
