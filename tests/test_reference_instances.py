"""The reference's own instances, on the CPU: the Netlib LPs of its tree (data/netlib/*.mps)
and the 120 generated instances of its cross-engine gate (tests/unit/test_pdhg.cpp:178-222).

* The committed fixtures (tests/golden/netlib.npz, tests/golden/kkt_fuzz_120.npz) hold exactly
  what the reference's MPS reader and test generator produce (checked where the reference
  build exists).
* The oracle (the C restatement) meets the gate's bar on all 120 instances: optimal at
  pdhg_tolerance 1e-9 with the objective within 1e-6 of the analytic optimum, and equal to
  what the reference's solve_pdhg returned; on the Netlib LPs it returns the reference's
  status and objective.

The same instances run on the GPU in tests/test_gpu_reference_instances.py.
"""
import os

import numpy as np
import pytest

import oracle
from tests.cases import kkt_fuzz_cases, netlib_cases

REF_TREE = "/root/reference/data/netlib"
needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference build (oracle/_ref) not present")

FIELDS = ("col_starts", "row_indices", "values", "cost", "col_lower", "col_upper",
          "row_lower", "row_upper")


@needs_ref
@pytest.mark.skipif(not os.path.isdir(REF_TREE), reason="reference tree not present")
def test_netlib_fixture_is_what_the_reference_reader_reads():
    for lp, _, _, _ in netlib_cases():
        got = oracle.ref_read_model(os.path.join(REF_TREE, lp.name + ".mps"))
        assert (got.num_rows, got.num_cols, got.maximize) == (lp.num_rows, lp.num_cols,
                                                               lp.maximize)
        for k in FIELDS:
            assert np.array_equal(getattr(got, k), getattr(lp, k)), (lp.name, k)
        assert got.objective_offset == lp.objective_offset


@needs_ref
def test_fuzz_fixture_is_what_the_reference_generator_draws():
    cases = kkt_fuzz_cases()
    assert len(cases) == 120
    for k in (0, 1, 7, 59, 119):
        lp = cases[k][0]
        got = oracle.ref_kkt_instance(20260904, 6, 6, k)
        for f in FIELDS:
            assert np.array_equal(getattr(got, f), getattr(lp, f)), (k, f)
        assert got.optimal_objective == lp.optimal_objective


def test_oracle_meets_the_cross_engine_gate_on_all_120():
    compared = 0
    for lp, ref_status, ref_objective in kkt_fuzz_cases():
        o = oracle.oracle_solve(lp, tolerance=1e-9, iteration_limit=1000000)
        assert o.status == ref_status, (lp.name, o.status, ref_status)
        if o.status != "optimal":
            continue
        compared += 1
        scale = max(1.0, abs(lp.optimal_objective))
        assert abs(o.objective - lp.optimal_objective) <= 1e-6 * scale, lp.name
        assert o.objective == ref_objective, (lp.name, o.objective, ref_objective)
    assert compared > 60


@pytest.mark.parametrize("case", netlib_cases()[:5], ids=lambda c: c[0].name)
def test_oracle_returns_the_reference_answer_on_netlib(case):
    lp, published, ref_status, ref_objective = case
    o = oracle.oracle_solve(lp, tolerance=1e-8, iteration_limit=1000000)
    assert o.status == ref_status
    assert o.objective == ref_objective
    if ref_status == "optimal":
        assert abs(o.objective - published) <= 1e-6 * max(1.0, abs(published))
