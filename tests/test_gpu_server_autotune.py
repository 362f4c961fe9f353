"""The served engine's chunk autotuner (sankhya_pdhg_server_config.chunk_attempts = -1).

Chunking only decides where an LP pauses between launches, never what it computes, so a
server that searches its chunk length for the most work per second must return, for every
LP, the bits the one-launch batched solve returns. The length it settles on is stored in the
autotune cache under the family of the admitted LPs (their nonzero and row statistics), and a
server on a family with a cached length uses it.
"""
import numpy as np
import pytest

from sih26_b200 import lpgen
from sih26_b200 import pdhg as P

pytestmark = pytest.mark.gpu


def _family():
    return lpgen.uneven_batch(count=96, m_lo=50, m_hi=400, infeasible_fraction=0.1, seed=11)


def _opts():
    return P.Options(pdhg_tolerance=1e-6, iteration_limit=200000, pdhg_algorithm="halpern",
                     pdhg_stop_rule="relative_kkt")


def test_autotuned_chunks_change_no_answer_and_the_cache_is_read(tmp_path, monkeypatch):
    cache = tmp_path / "autotune.tsv"
    monkeypatch.setenv("SANKHYA_PDHG_AUTOTUNE_CACHE", str(cache))
    lps = _family()
    want = P.batch_solve(lps, _opts())
    with P.Server(chunk_attempts=-1) as srv:
        got = srv.solve_all(lps, _opts())
        st = srv.stats()
    assert st["chunk_source"] == "tuned" and 16 <= st["chunk_attempts"] <= 8192, st
    assert st["rounds"] > 0 and st["family"].startswith("served|"), st
    for lp, a, b in zip(lps, got, want):
        assert a.status == b.status and a.iterations == b.iterations, lp.name
        assert np.array_equal(a.col_value, b.col_value), lp.name
        assert np.array_equal(a.row_dual, b.row_dual), lp.name
    if cache.exists():  # the search settled within the run and stored its pick
        for line in cache.read_text().splitlines():
            key, chunk, _ = line.split("\t")
            assert key == st["family"] and 16 <= int(chunk) <= 8192, line

    # a chunk cached for the family is where the next server starts (the last line wins)
    with open(cache, "a") as f:
        f.write(f"{st['family']}\t777\t0\n")
    with P.Server(chunk_attempts=-1) as srv:
        got2 = srv.solve_all(lps, _opts())
        st2 = srv.stats()
    assert st2["chunk_source"] == "cache" and st2["chunk_attempts"] == 777, st2
    for lp, a, b in zip(lps, got2, want):
        assert a.status == b.status and a.iterations == b.iterations, lp.name
        assert np.array_equal(a.col_value, b.col_value), lp.name


def test_a_configured_chunk_is_left_alone(tmp_path, monkeypatch):
    monkeypatch.setenv("SANKHYA_PDHG_AUTOTUNE_CACHE", str(tmp_path / "autotune.tsv"))
    lps = _family()[:40]
    with P.Server(chunk_attempts=300) as srv:
        srv.solve_all(lps, _opts())
        st = srv.stats()
    assert st["chunk_source"] == "configured" and st["chunk_attempts"] == 300, st
    assert not (tmp_path / "autotune.tsv").exists()
