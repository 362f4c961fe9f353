"""TEST INFRASTRUCTURE ONLY: Solution::recompute_quality restated in numpy.

Follows src/core/model.cpp:228-424 (the reference's measurement of a reported point) term by
term and in its order of summation: row activities accumulate column by column
(SparseMatrix::multiply, src/la/sparse.cpp:202-212), each column's a_j'row_dual down the
column in row order, the objective from the offset in column order
(Model::evaluate_objective, src/core/model.cpp:99-105). Every other figure is a maximum, so
its order does not matter. Pinned to the reference build by tests/test_quality_oracle.py; the
GPU path's quality block is checked against it.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

INF_BOUND = 1e30


def _finite(v):
    return np.abs(v) < INF_BOUND


def _minus_column_terms(start, cs, ri, vals, vec):
    """start_j - vals[k] * vec[ri[k]] for every entry k of column j, one after another in
    storage order (sequential within each column, all columns at once)."""
    n = len(cs) - 1
    lens = np.diff(cs)
    out = np.array(start, dtype=np.float64, copy=True)
    for t in range(int(lens.max()) if n else 0):
        cols = np.nonzero(lens > t)[0]
        k = cs[cols] + t
        out[cols] -= vals[k] * vec[ri[k]]
    return out


def _sequential(start, terms):
    acc = float(start)
    for t in terms:
        acc += float(t)
    return acc


def recompute_quality(lp, x, row_dual, col_dual, dual_bound) -> dict:
    m, n = lp.num_rows, lp.num_cols
    cs = np.asarray(lp.col_starts, dtype=np.int64)
    ri = np.asarray(lp.row_indices, dtype=np.int64)
    vals = np.asarray(lp.values, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64)
    row_dual = np.asarray(row_dual, dtype=np.float64)
    col_dual = np.asarray(col_dual, dtype=np.float64)
    cost = np.asarray(lp.cost, dtype=np.float64)
    cl, cu = np.asarray(lp.col_lower, float), np.asarray(lp.col_upper, float)
    rl, ru = np.asarray(lp.row_lower, float), np.asarray(lp.row_upper, float)
    col_of = np.repeat(np.arange(n), np.diff(cs))

    # :233-235 row activities, column by column (scipy's CSC product scatters in that order)
    act = (sp.csc_matrix((vals, ri, cs), shape=(m, n)) @ x) if m else np.zeros(0)
    # :244-253 row term scale: max(1, max |a_ij x_j|) over x_j != 0
    row_scale = np.ones(m)
    nz = x[col_of] != 0.0
    np.maximum.at(row_scale, ri[nz], np.abs(vals[nz] * x[col_of[nz]]))

    primal = [0.0]
    primal_scaled = [0.0]

    def record(viol, scale):
        keep = viol > 0.0
        if keep.any():
            primal.append(float(viol[keep].max()))
            primal_scaled.append(float((viol[keep] / np.maximum(1.0, scale[keep])).max()))

    fl, fu = _finite(cl), _finite(cu)
    record(np.where(fl, cl - x, 0.0), np.abs(x))
    record(np.where(fu, x - cu, 0.0), np.abs(x))
    frl, fru = _finite(rl), _finite(ru)
    record(np.where(frl, rl - act, 0.0), row_scale)
    record(np.where(fru, act - ru, 0.0), row_scale)

    objective = _sequential(lp.objective_offset, cost * x)

    sense = -1.0 if lp.maximize else 1.0
    dual = [0.0]
    dual_scaled = [0.0]
    comp = [0.0]
    dual_norm = float(np.abs(row_dual).max()) if m else 0.0

    # :301-310 column scale: max(1, |c_j|, max_i |a_ij row_dual_i|)
    terms = np.abs(cost).copy()
    np.maximum.at(terms, col_of, np.abs(vals * row_dual[ri]))
    col_scale = np.maximum(1.0, terms)

    def record_dual(viol, scale):
        keep = viol > 0.0
        if keep.any():
            dual.append(float(viol[keep].max()))
            dual_scaled.append(float((viol[keep] / scale[keep]).max()))

    def nearest(v, lo, hi):
        d = np.full(len(v), np.inf)
        f = _finite(lo)
        d[f] = np.minimum(d[f], np.abs(v[f] - lo[f]))
        f = _finite(hi)
        d[f] = np.minimum(d[f], np.abs(v[f] - hi[f]))
        return d

    def record_comp(mult, slack, mult_scale, primal_scale):
        keep = (mult != 0.0) & _finite(slack)
        if keep.any():
            prod = mult[keep] * slack[keep]
            comp.append(float(prod.max()))
            dual_scaled.append(float((prod / np.maximum(
                1.0, mult_scale[keep] * primal_scale[keep])).max()))

    # :360-378 consistency of col_dual with c - A'row_dual (pure LP)
    implied = _minus_column_terms(cost, cs, ri, vals, row_dual)
    record_dual(np.abs(implied - col_dual), np.maximum(1.0, terms))

    # :380-396 columns
    free = cl != cu
    d = sense * col_dual
    record_dual(np.where(free & (d > 0.0) & ~fl, d, 0.0), col_scale)
    record_dual(np.where(free & (d < 0.0) & ~fu, -d, 0.0), col_scale)
    record_comp(np.where(free, np.abs(d), 0.0), nearest(x, cl, cu), col_scale,
                np.maximum(1.0, np.abs(x)))

    # :404-416 rows
    y = sense * row_dual
    rfree = rl != ru
    price = np.full(m, max(1.0, dual_norm))
    record_dual(np.where(rfree & (y > 0.0) & ~frl, y, 0.0), price)
    record_dual(np.where(rfree & (y < 0.0) & ~fru, -y, 0.0), price)
    record_comp(np.where(rfree, np.abs(y), 0.0), nearest(act, rl, ru), price, row_scale)

    absolute_gap = abs(objective - dual_bound)
    return {
        "primal_infeasibility": max(primal),
        "primal_infeasibility_scaled": max(primal_scaled),
        "dual_infeasibility": max(dual),
        "dual_infeasibility_scaled": max(dual_scaled),
        "complementarity_violation": max(comp),
        "objective": objective,
        "absolute_gap": absolute_gap,
        "relative_gap": absolute_gap / max(1.0, abs(objective)),
    }
