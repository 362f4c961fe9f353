"""Scaling and layout on the device (prep_kernels.cuh) against the host code (pdhg_host.cpp,
itself bit-identical to the reference's build_scaling): the two preparations must give the same
bits, so every solve takes the same path -- same iteration count, same point, to the last bit."""
import math

import numpy as np
import pytest

from cases import hand_cases
from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = pytest.mark.gpu


def _both(lp, **kw):
    out = []
    for where in ("host", "device"):
        o = P.Options(pdhg_tolerance=1e-6, iteration_limit=3000, pdhg_prep=where)
        for k, v in kw.items():
            o.set(k, v)
        out.append(P.solve_pdhg(lp, o))
    return out


def _same(a, b):
    assert a.status == b.status and a.iterations == b.iterations, (a.status, b.status,
                                                                     a.iterations, b.iterations)
    assert a.spectral_norm == b.spectral_norm
    assert np.array_equal(a.col_value, b.col_value)
    assert np.array_equal(a.row_dual, b.row_dual)
    assert np.array_equal(a.col_dual, b.col_dual)


def _with_empty_row_and_column(lp):
    """An extra row with no entries (free) and an extra column with no entries (boxed)."""
    n = lp.num_cols
    cs = np.concatenate([lp.col_starts, [lp.col_starts[-1]]]).astype(np.int32)
    return lpgen.LP(num_rows=lp.num_rows + 1, num_cols=n + 1, col_starts=cs,
                    row_indices=lp.row_indices, values=lp.values,
                    cost=np.concatenate([lp.cost, [1.0]]),
                    col_lower=np.concatenate([lp.col_lower, [0.0]]),
                    col_upper=np.concatenate([lp.col_upper, [2.0]]),
                    row_lower=np.concatenate([lp.row_lower, [-math.inf]]),
                    row_upper=np.concatenate([lp.row_upper, [math.inf]]), name="with-empties")


CASES = [
    ("powerlaw_20k", lambda: lpgen.powerlaw_planted(m=20000, n=50000, seed=3)),
    ("uniform_2000x5000", lambda: lpgen.uniform_planted(2000, 5000, 10, seed=1)),
    ("blockangular_small", lambda: lpgen.block_angular_planted(blocks=4, block_rows=400,
                                                               block_cols=1000, linking_rows=40,
                                                               seed=5)),
    ("empties", lambda: _with_empty_row_and_column(lpgen.uniform_planted(60, 150, 4, seed=2))),
]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_preparation_gives_the_host_bits(name, make, precision):
    a, b = _both(make(), pdhg_precision=precision)
    _same(a, b)


@pytest.mark.parametrize("name,lp,expected", hand_cases())
def test_device_preparation_on_the_hand_lps(name, lp, expected):
    a, b = _both(lp, pdhg_tolerance=1e-8, iteration_limit=200000)
    _same(a, b)
    assert b.status == "optimal", b.message
