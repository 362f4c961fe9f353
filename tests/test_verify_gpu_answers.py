"""Every committed GPU answer passes the reference's independent verifier.

tests/golden/gpu_answers/ holds answers the GPU engine returned (made on a B200 by
tests/golden/make_gpu_answers.py) as the reference's model and solution files: optimal
points of the parity LPs, the Netlib LPs and a batched sample, Farkas certificates of
infeasible LPs and rays of unbounded ones. The reference's tools/verify_solution.py
(tools/verify_solution.py:718 verify, :562 verify_farkas, :639 verify_ray, :1150 main), which
shares no code with any solver, must print VERIFIED and exit 0 on each. It runs where the
reference tree exists (this test reads it from there and never copies it).

tests/test_gpu_answers_current.py keeps the committed answers tied to the current GPU code.
"""
import glob
import os
import subprocess
import sys

import pytest

VERIFIER = "/root/reference/tools/verify_solution.py"
ANSWERS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "gpu_answers")
PAIRS = sorted(glob.glob(os.path.join(ANSWERS, "*.sol.gz")))

needs_tree = pytest.mark.skipif(not os.path.exists(VERIFIER),
                                reason="the reference's verifier is not present")


def test_answers_are_committed():
    assert len(PAIRS) >= 60, len(PAIRS)


@needs_tree
@pytest.mark.parametrize("sol", PAIRS, ids=lambda p: os.path.basename(p)[:-7])
def test_reference_verifier_accepts(sol):
    model = sol[:-len(".sol.gz")] + ".mps.gz"
    p = subprocess.run([sys.executable, VERIFIER, model, sol], capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-2000:]
    assert "VERIFIED" in p.stdout
