"""Seeded synthetic LPs with a planted primal-dual optimum.

These stand in for the LP families the reference benchmarks its restarted PDHG on (its
own planted generator is bench/runners/generate_large_lp.py:49-206; the fuzz family is
tests/oracles/lp_generator.cpp:122-189). Every instance is built backwards from a chosen
KKT point, so its optimal objective is known before anything is solved:

    min c'x  s.t.  row_lower <= A x <= row_upper,  col_lower <= x <= col_upper

    x*     30 % at the lower bound 0, 10 % at the upper bound u ~ U(1, 10), the rest U(0, u)
    lam*   row multipliers (simplex sign: c = A' lam* + z*); equality rows lam* ~ N(0, 1)
    z*     reduced costs complementary to x*: +U(0.1, 1) at lower, -U(0.1, 1) at upper, else 0
    c      = A' lam* + z*
    rows   equality rows b = A x*; an inequality row is tight (lam* of the right sign) or slack
           (lam* = 0) at x*

The matrix is held the way the reference holds it (include/sankhya/sparse.hpp:109-112): CSC,
int32 column starts and row indices, rows ascending inside each column, FP64 values.

All randomness comes from numpy's PCG64 seeded by `seed`, so a (family, seed) pair fixes
every draw. scipy.sparse is used only to sort COO triplets into CSC.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional

import numpy as np

INF = float("inf")


@dataclasses.dataclass
class LP:
    """One LP in the reference's Model layout (include/sankhya/model.hpp:131-225)."""

    num_rows: int
    num_cols: int
    col_starts: np.ndarray  # int32 [n+1]
    row_indices: np.ndarray  # int32 [nnz]
    values: np.ndarray  # float64 [nnz]
    cost: np.ndarray  # float64 [n], in the model's own sense
    col_lower: np.ndarray
    col_upper: np.ndarray
    row_lower: np.ndarray
    row_upper: np.ndarray
    maximize: bool = False
    objective_offset: float = 0.0
    name: str = ""
    # planted optimum (None for instances without one)
    x_star: Optional[np.ndarray] = None
    row_dual_star: Optional[np.ndarray] = None
    optimal_objective: Optional[float] = None
    # a Farkas ray when the instance was made infeasible on purpose
    farkas_star: Optional[np.ndarray] = None
    # a primal ray when the instance was made unbounded on purpose
    ray_star: Optional[np.ndarray] = None
    # a quadratic objective 0.5 x'Qx: Q's lower triangle in CSC (include/sankhya/model.hpp:156)
    hessian_col_starts: Optional[np.ndarray] = None
    hessian_row_indices: Optional[np.ndarray] = None
    hessian_values: Optional[np.ndarray] = None

    @property
    def num_nonzeros(self) -> int:
        return int(self.col_starts[-1])

    def check(self) -> None:
        """Structural checks the CUDA path relies on (indices in range, sorted, sizes)."""
        n, m = self.num_cols, self.num_rows
        cs = self.col_starts
        assert cs.dtype == np.int32 and cs.shape == (n + 1,) and cs[0] == 0
        assert np.all(np.diff(cs.astype(np.int64)) >= 0)
        assert self.row_indices.dtype == np.int32 and self.row_indices.shape == (cs[-1],)
        assert self.values.dtype == np.float64 and self.values.shape == (cs[-1],)
        if cs[-1]:
            assert self.row_indices.min() >= 0 and self.row_indices.max() < m
        for a in (self.cost, self.col_lower, self.col_upper):
            assert a.dtype == np.float64 and a.shape == (n,)
        for a in (self.row_lower, self.row_upper):
            assert a.dtype == np.float64 and a.shape == (m,)

    def to_scipy_csc(self):
        import scipy.sparse as sp

        return sp.csc_matrix((self.values, self.row_indices, self.col_starts),
                             shape=(self.num_rows, self.num_cols))


def _csc_from_coo(m: int, n: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray):
    import scipy.sparse as sp

    a = sp.coo_matrix((vals, (rows, cols)), shape=(m, n)).tocsc()
    a.sum_duplicates()
    a.sort_indices()
    return (a.indptr.astype(np.int32), a.indices.astype(np.int32),
            a.data.astype(np.float64))


def _distinct_rows_per_column(rng: np.random.Generator, m: int, n: int, k: int,
                              cdf: Optional[np.ndarray] = None) -> np.ndarray:
    """k distinct rows for each of n columns, uniform or by the row distribution `cdf`.

    Drawn with replacement and redrawn where a column repeats a row, which samples without
    replacement (each column's set is distinct, its law conditional on distinctness)."""
    assert k <= m

    def draw(size):
        if cdf is None:
            return rng.integers(0, m, size=size, dtype=np.int64)
        return np.minimum(np.searchsorted(cdf, rng.random(size), side="right"), m - 1)

    rows = draw((n, k))
    while True:
        rows.sort(axis=1)
        dup = np.zeros(rows.shape, dtype=bool)
        dup[:, 1:] = rows[:, 1:] == rows[:, :-1]
        if not dup.any():
            return rows
        rows[dup] = draw(int(dup.sum()))


def _plant(rng: np.random.Generator, a_csc, m: int, n: int, row_kind: np.ndarray,
           upper_lo: float = 1.0, upper_hi: float = 10.0):
    """Choose x*, lam*, z* and derive c and the row bounds (module docstring).

    row_kind: 0 equality, 1 '<=' tight, 2 '<=' slack."""
    u = rng.uniform(upper_lo, upper_hi, n)
    pick = rng.random(n)
    at_lower = pick < 0.3
    at_upper = (pick >= 0.3) & (pick < 0.4)
    x = rng.uniform(0.0, 1.0, n) * u
    x[at_lower] = 0.0
    x[at_upper] = u[at_upper]
    z = np.zeros(n)
    mag = rng.uniform(0.1, 1.0, n)
    z[at_lower] = mag[at_lower]
    z[at_upper] = -mag[at_upper]
    lam = rng.standard_normal(m)
    tight_le = row_kind == 1
    slack_le = row_kind == 2
    lam[tight_le] = -rng.uniform(0.1, 1.0, int(tight_le.sum()))
    lam[slack_le] = 0.0
    ax = a_csc @ x
    c = a_csc.T @ lam + z
    row_lower = ax.copy()
    row_upper = ax.copy()
    row_lower[tight_le | slack_le] = -INF
    slack = rng.uniform(0.1, 1.0, m) * (1.0 + np.abs(ax))
    row_upper[slack_le] = ax[slack_le] + slack[slack_le]
    return x, lam, c, np.zeros(n), u, row_lower, row_upper


def _assemble(name, m, n, cs, ri, vals, rng, row_kind, **kw) -> LP:
    import scipy.sparse as sp

    a = sp.csc_matrix((vals, ri, cs), shape=(m, n))
    x, lam, c, lo, up, rl, ru = _plant(rng, a, m, n, row_kind, **kw)
    lp = LP(num_rows=m, num_cols=n, col_starts=cs, row_indices=ri, values=vals, cost=c,
            col_lower=lo, col_upper=up, row_lower=rl, row_upper=ru, name=name, x_star=x,
            row_dual_star=lam, optimal_objective=float(c @ x))
    lp.check()
    return lp


def uniform_planted(m: int, n: int, nnz_per_col: int, seed: int, name: str = "") -> LP:
    """The single-LP family of 2,000 x 5,000 with 10 nonzeros per column: uniform distinct
    rows per column, N(0,1) values, equality rows, 0 <= x <= u, planted optimum."""
    rng = np.random.default_rng(seed)
    rows = _distinct_rows_per_column(rng, m, n, nnz_per_col)
    vals = rng.standard_normal((n, nnz_per_col))
    cs = (np.arange(n + 1, dtype=np.int64) * nnz_per_col).astype(np.int32)
    return _assemble(name or f"uniform-{m}x{n}-s{seed}", m, n, cs, rows.astype(np.int32).ravel(),
                     vals.ravel(), rng, np.zeros(m, dtype=np.int8))


def powerlaw_planted(m: int = 200_000, n: int = 500_000, nnz_per_col: int = 10,
                     alpha: float = 1.5, seed: int = 1, name: str = "") -> LP:
    """The skewed single-LP family (200,000 x 500,000, about 5M nonzeros): each column's
    rows drawn by Pareto(alpha) row weights so a few rows hold thousands of entries; values
    N(0,1) times a per-row factor 10^U(-2,2); equality rows; planted optimum."""
    rng = np.random.default_rng(seed)
    w = (1.0 - rng.random(m)) ** (-1.0 / alpha)
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    rows = _distinct_rows_per_column(rng, m, n, nnz_per_col, cdf)
    row_factor = 10.0 ** rng.uniform(-2.0, 2.0, m)
    vals = rng.standard_normal((n, nnz_per_col)) * row_factor[rows]
    cs = (np.arange(n + 1, dtype=np.int64) * nnz_per_col).astype(np.int32)
    return _assemble(name or f"powerlaw-{m}x{n}-s{seed}", m, n, cs,
                     rows.astype(np.int32).ravel(), vals.ravel(), rng,
                     np.zeros(m, dtype=np.int8))


def block_angular_planted(blocks: int = 64, block_rows: int = 4_000, block_cols: int = 10_000,
                          nnz_per_col: int = 8, linking_rows: int = 2_000,
                          linking_density: float = 0.02, le_fraction: float = 0.3,
                          seed: int = 2, name: str = "") -> LP:
    """The blending-style block-angular family: `blocks` diagonal blocks of block_rows x
    block_cols with nnz_per_col entries per column, values U(0.1, 2) with 20 % negated, plus
    dense-ish linking rows each touching `linking_density` of all columns; 30 % of rows are
    '<=' (tight or slack at x*), the rest equalities; planted optimum."""
    rng = np.random.default_rng(seed)
    n = blocks * block_cols
    m = blocks * block_rows + linking_rows
    local = _distinct_rows_per_column(rng, block_rows, n, nnz_per_col)
    block_of_col = np.arange(n) // block_cols
    brow = (local + (block_of_col * block_rows)[:, None]).ravel()
    bcol = np.repeat(np.arange(n), nnz_per_col)
    per_link = int(round(linking_density * n))
    lcols = _distinct_rows_per_column(rng, n, linking_rows, per_link).ravel()
    lrow = np.repeat(np.arange(linking_rows) + blocks * block_rows, per_link)
    rows = np.concatenate([brow, lrow])
    cols = np.concatenate([bcol, lcols])
    vals = rng.uniform(0.1, 2.0, rows.size)
    vals[rng.random(rows.size) < 0.2] *= -1.0
    cs, ri, v = _csc_from_coo(m, n, rows, cols, vals)
    kind = np.zeros(m, dtype=np.int8)
    le = rng.random(m) < le_fraction
    tight = rng.random(m) < 0.5
    kind[le & tight] = 1
    kind[le & ~tight] = 2
    return _assemble(name or f"blockangular-{m}x{n}-s{seed}", m, n, cs, ri, v, rng, kind)


def small_planted(m: int, n: int, nnz_lo: int, nnz_hi: int, rng: np.random.Generator,
                  name: str = "") -> LP:
    """One LP of the uneven batch family: nnz per column uniform on [nnz_lo, nnz_hi]
    (capped at m), uniform distinct rows, N(0,1) values, equality rows, planted optimum."""
    k = np.minimum(rng.integers(nnz_lo, nnz_hi + 1, n), m)
    kmax = int(k.max())
    rows = _distinct_rows_per_column(rng, m, n, kmax)
    # keep the first k_j of each column's kmax distinct rows (a random subset, then sorted)
    order = np.argsort(rng.random((n, kmax)), axis=1)
    rows = np.take_along_axis(rows, order, axis=1)
    keep = np.arange(kmax)[None, :] < k[:, None]
    cols = np.repeat(np.arange(n), kmax).reshape(n, kmax)[keep]
    rr = rows[keep]
    vals = rng.standard_normal(rr.size)
    cs, ri, v = _csc_from_coo(m, n, rr, cols, vals)
    return _assemble(name, m, n, cs, ri, v, rng, np.zeros(m, dtype=np.int8))


def make_infeasible(lp: LP, rng: np.random.Generator, margin: float = 0.1) -> LP:
    """Shift b off the range of A over the box so a Farkas certificate exists by
    construction: draw y_hat, then b <- b + t*y_hat with t chosen so that
    y_hat'b exceeds max over the box of (A'y_hat)'x by a margin (equality rows)."""
    a = lp.to_scipy_csc()
    y_hat = rng.standard_normal(lp.num_rows)
    g = a.T @ y_hat
    box_max = float(np.sum(np.where(g > 0, g * lp.col_upper, g * lp.col_lower)))
    b = lp.row_lower.copy()
    target = box_max + margin * (1.0 + abs(box_max))
    t = max(target - float(y_hat @ b), 0.0) / float(y_hat @ y_hat)
    b = b + t * y_hat
    out = dataclasses.replace(lp, row_lower=b.copy(), row_upper=b.copy(), x_star=None,
                              row_dual_star=None, optimal_objective=None,
                              name=lp.name + "-infeasible")
    out.farkas_star = y_hat
    return out


def make_unbounded(lp: LP, rng: np.random.Generator) -> LP:
    """Append two columns with no upper bound whose matrix columns cancel (a and -a, a the
    column of a random existing column) and whose costs sum to a negative number: moving both
    up together keeps every row activity and lowers the cost without limit, so a primal ray
    (0, ..., 0, 1, 1) exists by construction and the LP is unbounded."""
    j = int(rng.integers(0, lp.num_cols))
    b, e = int(lp.col_starts[j]), int(lp.col_starts[j + 1])
    rows = lp.row_indices[b:e]
    vals = lp.values[b:e]
    nnz = lp.num_nonzeros
    cs = np.concatenate([lp.col_starts, [nnz + rows.size, nnz + 2 * rows.size]]).astype(np.int32)
    ri = np.concatenate([lp.row_indices, rows, rows]).astype(np.int32)
    v = np.concatenate([lp.values, vals, -vals])
    c1 = -float(rng.uniform(0.5, 1.5))
    c2 = float(rng.uniform(0.0, 0.4))
    n = lp.num_cols + 2
    ray = np.zeros(n)
    ray[-2:] = 1.0
    out = dataclasses.replace(
        lp, num_cols=n, col_starts=cs, row_indices=ri, values=v,
        cost=np.concatenate([lp.cost, [c1, c2]]),
        col_lower=np.concatenate([lp.col_lower, [0.0, 0.0]]),
        col_upper=np.concatenate([lp.col_upper, [INF, INF]]), x_star=None, row_dual_star=None,
        optimal_objective=None, name=lp.name + "-unbounded")
    out.ray_star = ray
    out.check()
    return out


def qp_planted(m: int, n: int, nnz_per_col: int, seed: int, maximize: bool = False,
               name: str = "") -> LP:
    """A convex QP with a planted optimum: the LP family of uniform_planted plus
    Q = diag(d) + B'B (d ~ U(0.1, 1), B sparse with two N(0, 0.5^2) entries per row), stored
    as its lower triangle; c = A'lam + z - Q x* makes (x*, lam, z) a KKT point, so x* is optimal.
    With maximize the model is stated as max -(c'x + 0.5 x'Qx), the same problem."""
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    rows = _distinct_rows_per_column(rng, m, n, nnz_per_col)
    cols = np.repeat(np.arange(n), nnz_per_col)
    vals = rng.standard_normal(rows.size)
    cs, ri, v = _csc_from_coo(m, n, rows.ravel(), cols, vals)
    a = sp.csc_matrix((v, ri, cs), shape=(m, n))
    k = max(1, n // 2)
    b_rows = np.repeat(np.arange(k), 2)
    b_cols = rng.integers(0, n, size=2 * k)
    b = sp.coo_matrix((0.5 * rng.standard_normal(2 * k), (b_rows, b_cols)), shape=(k, n)).tocsc()
    q = (sp.diags(rng.uniform(0.1, 1.0, n)) + (b.T @ b)).tocsc()
    low = sp.tril(q).tocsc()
    low.sum_duplicates()
    low.sort_indices()
    x, lam, c_lin, lo, up, rl, ru = _plant(rng, a, m, n, np.zeros(m, dtype=np.int8))
    # _plant set c = A'lam + z for the LP; the QP's gradient adds Q x*
    c = c_lin - q @ x
    sense = -1.0 if maximize else 1.0
    lp = LP(num_rows=m, num_cols=n, col_starts=cs, row_indices=ri, values=v, cost=sense * c,
            col_lower=lo, col_upper=up, row_lower=rl, row_upper=ru, maximize=maximize,
            name=name or f"qp-{m}x{n}-s{seed}", x_star=x, row_dual_star=lam,
            optimal_objective=float(sense * (c @ x + 0.5 * x @ (q @ x))))
    lp.hessian_col_starts = low.indptr.astype(np.int32)
    lp.hessian_row_indices = low.indices.astype(np.int32)
    lp.hessian_values = (sense * low.data).astype(np.float64)
    lp.check()
    return lp


def uneven_batch(count: int = 512, m_lo: int = 50, m_hi: int = 5_000,
                 infeasible_fraction: float = 0.1, seed: int = 3) -> list[LP]:
    """The batched family: `count` LPs with m log-uniform on [m_lo, m_hi], n = round(m *
    U(1.5, 3)), 5-15 nonzeros per column, N(0,1) values, planted optimum; a fraction made
    primal-infeasible with a Farkas certificate by construction."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        m = int(round(math.exp(rng.uniform(math.log(m_lo), math.log(m_hi)))))
        n = int(round(m * rng.uniform(1.5, 3.0)))
        lp = small_planted(m, n, 5, 15, rng, name=f"batch{k}-{m}x{n}")
        if rng.random() < infeasible_fraction:
            lp = make_infeasible(lp, rng)
        out.append(lp)
    return out


def served_request(index: int, seed: int = 5, m_lo: int = 100, m_hi: int = 50_000,
                   infeasible_fraction: float = 0.1) -> LP:
    """Request `index` of the served stream: one LP drawn like the batched family but with m
    log-uniform on [m_lo, m_hi], from its own seeded generator (seed, index), so every request
    is a fresh LP and any request can be drawn without the ones before it."""
    rng = np.random.default_rng([seed, index])
    m = int(round(math.exp(rng.uniform(math.log(m_lo), math.log(m_hi)))))
    n = int(round(m * rng.uniform(1.5, 3.0)))
    lp = small_planted(m, n, 5, 15, rng, name=f"request{index}-{m}x{n}")
    if rng.random() < infeasible_fraction:
        lp = make_infeasible(lp, rng)
    return lp


def from_dense(rows, row_lower, row_upper, cost, col_lower=None, col_upper=None,
               maximize=False, objective_offset=0.0, name="") -> LP:
    """A tiny LP written out by hand, the way the reference's unit tests build them
    (tests/unit/test_pdhg.cpp:69-91): zero entries are not stored; default bounds
    0 <= x < inf."""
    a = np.asarray(rows, dtype=np.float64).reshape(len(row_lower), len(cost))
    m, n = a.shape
    cs = [0]
    ri, vals = [], []
    for j in range(n):
        for i in range(m):
            if a[i, j] != 0.0:
                ri.append(i)
                vals.append(a[i, j])
        cs.append(len(ri))
    lp = LP(num_rows=m, num_cols=n, col_starts=np.array(cs, dtype=np.int32),
            row_indices=np.array(ri, dtype=np.int32), values=np.array(vals, dtype=np.float64),
            cost=np.asarray(cost, dtype=np.float64),
            col_lower=np.zeros(n) if col_lower is None else np.asarray(col_lower, np.float64),
            col_upper=np.full(n, INF) if col_upper is None else np.asarray(col_upper, np.float64),
            row_lower=np.asarray(row_lower, dtype=np.float64),
            row_upper=np.asarray(row_upper, dtype=np.float64), maximize=maximize,
            objective_offset=objective_offset, name=name)
    lp.check()
    return lp
