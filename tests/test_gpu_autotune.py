"""The SpMV-schedule autotuner: candidates timed on the LP itself, keyed on row-length
statistics, cached on disk; a cached pick is reused and gives the same bits as the run that
measured it, and the answer meets the request either way."""
import os

import numpy as np
import pytest

import oracle
from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = pytest.mark.gpu

CANDIDATES = {(32, 16), (16, 16), (32, 8), (32, 32), (8, 16), (16, 8)}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_autotune_measures_then_reads_the_cache(tmp_path, monkeypatch, precision):
    cache = tmp_path / "autotune.tsv"
    monkeypatch.setenv("SANKHYA_PDHG_AUTOTUNE_CACHE", str(cache))
    lp = lpgen.powerlaw_planted(m=3000, n=7500, seed=4)
    opts = P.Options(pdhg_tolerance=1e-6, pdhg_stop_rule="relative_kkt", pdhg_autotune=True,
                     pdhg_precision=precision, pdhg_algorithm="halpern")
    first = P.solve_pdhg(lp, opts)
    assert first.autotuned == 1
    assert (first.schedule[0], first.schedule[1]) in CANDIDATES
    assert (first.schedule[2], first.schedule[3]) in CANDIDATES
    lines = cache.read_text().splitlines()
    assert len(lines) == 1 and "|rows:" in lines[0] and "|cols:" in lines[0]
    second = P.solve_pdhg(lp, opts)
    assert second.autotuned == 2 and second.schedule == first.schedule
    assert second.iterations == first.iterations
    assert np.array_equal(second.col_value, first.col_value)
    for s in (first, second):
        assert s.status in ("optimal", "feasible"), s.message
        r = oracle.oracle_evaluate(lp, s.col_value, -s.row_dual)
        assert max(r["primal"], r["dual"], r["gap"]) <= 1e-6


def test_fixed_rule_without_autotune(tmp_path, monkeypatch):
    monkeypatch.setenv("SANKHYA_PDHG_AUTOTUNE_CACHE", str(tmp_path / "none.tsv"))
    lp = lpgen.uniform_planted(200, 500, 5, seed=7)
    s = P.solve_pdhg(lp, P.Options(pdhg_tolerance=1e-6))
    assert s.autotuned == 0 and s.schedule == (32, 16, 32, 16)
    assert not os.path.exists(tmp_path / "none.tsv")
