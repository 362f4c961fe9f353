"""The committed GPU answers (tests/golden/gpu_answers/, judged by the reference's verifier in
tests/test_verify_gpu_answers.py) are what the current GPU code returns: every case of
tests/golden/make_gpu_answers.py is solved again and must give the committed status, and,
where a point is claimed, the committed objective to 1e-6."""
import gzip
import math
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_gpu_answers  # noqa: E402

pytestmark = pytest.mark.gpu


def _header(path):
    out = {}
    with gzip.open(path, "rt") as f:
        for line in f:
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            if line.startswith("begin"):
                break
            k, _, v = line.partition(" ")
            out[k] = v
    return out


def test_current_answers_match_the_committed_ones():
    cs = make_gpu_answers.cases()
    sols = make_gpu_answers.solve_all(cs)
    for (name, lp, _), s in zip(cs, sols):
        path = os.path.join(HERE, "golden", "gpu_answers", name + ".sol.gz")
        assert os.path.exists(path), name
        h = _header(path)
        assert s.status == h["status"], (name, s.status, h["status"])
        if s.status in ("optimal", "feasible"):
            want = float(h["objective"])
            assert math.isclose(s.objective, want, rel_tol=1e-6, abs_tol=1e-6), (name, s.objective,
                                                                                  want)
