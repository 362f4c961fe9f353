"""The CPU legs of bench.py that need no GPU: the reference sampled one LP per host core (the
batched and served CPU baselines) and the single-LP sample, on small LPs."""
import oracle
import pytest

import bench
from sih26_b200 import lpgen

needs_ref = pytest.mark.skipif(not oracle.ref_available(),
                               reason="reference build (oracle/_ref) not present")


@needs_ref
def test_cpu_batch_sample_charges_each_lp_its_iterations():
    lps = [lpgen.uniform_planted(40, 100, 4, seed=s) for s in (1, 2, 3)]
    few = bench.cpu_batch_sample(lps, [100, 100, 100], "three LPs")
    many = bench.cpu_batch_sample(lps, [100000, 100000, 100000], "three LPs")
    assert few["kind"] == "reference" and few["cores"] >= 1
    assert few["sample"].startswith("three LPs (3)")
    assert few["value"] > 0 and many["value"] > 0
    # a thousand times the iterations costs more than the setup-dominated sample
    assert many["cpu_seconds"] > few["cpu_seconds"]
    assert many["seconds"] >= max(many["cpu_seconds"] / many["cores"], 0.0) - 1e-12


@needs_ref
def test_cpu_reference_sample_times_setup_and_iterations():
    lp = lpgen.uniform_planted(60, 150, 4, seed=1)
    kind, threads, setup, per_it = bench.cpu_reference_sample(lp, 20)
    assert kind == "reference" and threads >= 1
    assert setup > 0 and per_it > 0
