"""The certificate checkers the GPU tests use, pinned to the reference's own
(src/core/certificate.cpp:29-218, through the reference build when it is present), on
certificates that exist by construction and on near-misses that must be turned down."""
import numpy as np
import pytest

import oracle
from certs import farkas_numpy, ray_numpy
from sih26_b200 import lpgen


def _infeasible(seed):
    rng = np.random.default_rng(seed)
    return lpgen.make_infeasible(lpgen.uniform_planted(40, 90, 4, seed=seed), rng)


def _unbounded(seed):
    rng = np.random.default_rng(seed)
    return lpgen.make_unbounded(lpgen.uniform_planted(40, 90, 4, seed=seed), rng)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_planted_farkas_certificate_and_near_misses(seed):
    lp = _infeasible(seed)
    y = lp.farkas_star
    cases = [(y, True), (-y, False), (np.zeros_like(y), False), (1e-3 * y, True)]
    for cert, want in cases:
        got, why = farkas_numpy(lp, cert)
        assert got == want, why
        if oracle.ref_available():
            ref, rwhy = oracle.ref_farkas_check(lp, cert)
            assert ref == want, rwhy


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_planted_primal_ray_and_near_misses(seed):
    lp = _unbounded(seed)
    d = lp.ray_star
    bent = d.copy()
    bent[0] = 0.5  # moves a bounded column: blocked either way by [0, u]
    half = d.copy()
    half[-1] = 0.0  # breaks the cancellation: row activity moves
    cases = [(d, True), (3.0 * d, True), (-d, False), (bent, False), (half, False),
             (np.zeros_like(d), False)]
    for cert, want in cases:
        got, why = ray_numpy(lp, cert)
        assert got == want, why
        if oracle.ref_available():
            ref, rwhy = oracle.ref_ray_check(lp, cert)
            assert ref == want, rwhy


def test_generators_keep_the_planted_structure():
    lp = _unbounded(4)
    assert lp.num_cols == 92 and np.isinf(lp.col_upper[-2:]).all()
    a = lp.to_scipy_csc()
    assert np.allclose(a @ lp.ray_star, 0.0)
    assert float(lp.cost @ lp.ray_star) < 0.0
