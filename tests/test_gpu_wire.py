"""Requests in the binary wire format (sankhya_pdhg_wire_*), solved on the GPU.

The wire format stands in for text MPS in served mode (the reference reads MPS/LP text,
src/io/mps_reader.cpp). A request buffer is viewed in place (sankhya_pdhg_wire_view: the
problem struct points into the buffer, nothing is copied on the host) and handed to the
single-LP solve and to the resident server. The answers must be bit-for-bit those of the
same LP passed as ordinary arrays, and their residuals, recomputed by the oracle from the
returned point, must meet the request.
"""
import math

import numpy as np
import pytest

import oracle
from sih26_b200 import lpgen
from sih26_b200 import pdhg as P
from tests.test_quality_oracle import edge_lps

pytestmark = pytest.mark.gpu


def _lps():
    out = [("uniform", lpgen.uniform_planted(300, 750, 6, seed=3)),
           ("maximise", lpgen.from_dense([[1, 0], [0, 2], [3, 2]], [-math.inf] * 3, [4, 12, 18],
                                         [3, 5], maximize=True, objective_offset=2.5)),
           ("block_angular", lpgen.block_angular_planted(blocks=3, block_rows=40, block_cols=100,
                                                         nnz_per_col=4, linking_rows=6, seed=4))]
    out += edge_lps()
    return out


def _same(a, b):
    assert a.status == b.status and a.iterations == b.iterations
    assert a.objective == b.objective or (math.isnan(a.objective) and math.isnan(b.objective))
    for f in ("col_value", "row_dual", "col_dual"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name,lp", _lps(), ids=[n for n, _ in _lps()])
def test_single_lp_from_a_wire_buffer_is_the_direct_solve(name, lp, precision):
    opts = P.Options(pdhg_tolerance=1e-7, iteration_limit=100000, pdhg_precision=precision,
                     pdhg_algorithm="halpern", pdhg_stop_rule="relative_kkt")
    req = P.WireRequest(P.to_wire(lp))
    via_wire = P.solve_wire(req, opts)
    direct = P.solve_pdhg(lp, opts)
    _same(via_wire, direct)
    if via_wire.status in ("optimal", "feasible"):
        sense = -1.0 if lp.maximize else 1.0
        r = oracle.oracle_evaluate(lp, via_wire.col_value, -sense * via_wire.row_dual)
        assert max(r["primal"], r["dual"], r["gap"]) <= 1e-7 * (1 + 1e-6), (name, r)


def test_server_takes_wire_requests():
    lps = [lp for _, lp in _lps()] + [lpgen.uniform_planted(80 + 20 * k, 200 + 40 * k, 4,
                                                            seed=50 + k) for k in range(6)]
    opts = P.Options(pdhg_tolerance=1e-6, iteration_limit=100000, pdhg_algorithm="halpern",
                     pdhg_stop_rule="relative_kkt")
    want = P.batch_solve(lps, opts)
    with P.Server() as srv:
        tickets = [srv.submit_wire(P.WireRequest(P.to_wire(lp)), opts) for lp in lps]
        done = {}
        for _ in range(100000):
            srv.step()
            for t in tickets:
                if t not in done:
                    r = srv.result(t)
                    if r is not None:
                        done[t] = r
            if len(done) == len(tickets):
                break
    assert len(done) == len(tickets)
    for lp, t, w in zip(lps, tickets, want):
        got = done[t]
        assert got.status == w.status and got.iterations == w.iterations, lp.name
        for f in ("col_value", "row_dual", "col_dual"):
            assert np.array_equal(getattr(got, f), getattr(w, f)), (lp.name, f)
