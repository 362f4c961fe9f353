"""The certificate checkers the GPU tests use, pinned to the reference's own
(src/core/certificate.cpp:29-218, through the reference build when it is present), on
certificates that exist by construction and on near-misses that must be turned down; and the
known answers of the reference's certificate tests (tests/unit/test_certificate.cpp:73-182) on
all three checkers: the numpy restatement, the reference's own, and the library's
farkas_holds / ray_holds that every certificate passes before the library reports it."""
import os

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


# The known answers of the reference's certificate tests (tests/unit/test_certificate.cpp:
# 73-182): (name, kind, A rows, row_lower, row_upper, cost, col_lower, col_upper, vector,
# verdict, a phrase of the reference checker's reason).
_INF = float("inf")
_PAIR = ([[1.0], [1.0]], [5.0, -_INF], [_INF, 2.0], [1.0], [0.0], [_INF])  # x >= 5, x <= 2
_OPEN = ([[1.0]], [1.0], [_INF], [-1.0], [-_INF], [_INF])  # min -x, x >= 1
KNOWN_ANSWERS = [
    ("aggregate_rows", "F", *_PAIR, [1.0, -1.0], True, "at least 3"),
    ("scaled_up", "F", *_PAIR, [1e6, -1e6], True, None),
    ("scaled_down", "F", *_PAIR, [1e-6, -1e-6], True, None),
    ("opposite_sign", "F", *_PAIR, [-1.0, 1.0], False, None),
    ("missing_row_bound", "F", *_PAIR, [-1.0, -1.0], False, "does not have"),
    ("free_column", "F", [[1.0]], [5.0], [_INF], [1.0], [-_INF], [_INF], [1.0], False,
     "free upward"),
    ("all_zero", "F", *_PAIR, [0.0, 0.0], False, "every multiplier is zero"),
    ("marginal", "F", [[1.0], [1.0]], [5.0, -_INF], [_INF, 5.0 - 1e-12], [1.0], [0.0], [_INF],
     [1.0, -1.0], False, "not a contradiction beyond rounding"),
    ("unblocked_ray", "R", *_OPEN, [1.0], True, "improves"),
    ("worsening_ray", "R", *_OPEN, [-1.0], False, None),
    ("bound_blocks", "R", [[1.0]], [1.0], [_INF], [-1.0], [-_INF], [10.0], [1.0], False,
     "upper bound"),
    ("row_blocks", "R", [[1.0, 1.0]], [-_INF], [10.0], [-1.0, -1.0], [-_INF, -_INF],
     [_INF, _INF], [1.0, 1.0], False, "row"),
    ("zero_direction", "R", *_OPEN, [0.0], False, "not a direction"),
]


def _known_lp(case):
    _, _, rows, rl, ru, cost, cl, cu, *_ = case
    return lpgen.from_dense(rows, rl, ru, cost, cl, cu)


@pytest.mark.parametrize("case", KNOWN_ANSWERS, ids=[c[0] for c in KNOWN_ANSWERS])
def test_numpy_and_reference_checkers_give_the_reference_known_answers(case):
    name, kind, *_, vec, want, phrase = case
    lp = _known_lp(case)
    got, why = (farkas_numpy if kind == "F" else ray_numpy)(lp, vec)
    assert got == want, (name, why)
    if oracle.ref_available():
        got, why = (oracle.ref_farkas_check if kind == "F" else oracle.ref_ray_check)(lp, vec)
        assert got == want, (name, why)
        if phrase:
            assert phrase in why, (name, why)


@pytest.fixture(scope="module")
def cert_checker(tmp_path_factory):
    """tests/certificate_check.cpp compiled against the library's host source."""
    import shutil
    import subprocess

    cuda_inc = "/usr/local/cuda/include"
    if shutil.which("g++") is None or not os.path.isdir(cuda_inc):
        pytest.skip("no C++ compiler or CUDA headers")
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    exe = tmp_path_factory.mktemp("certs") / "certificate_check"
    cmd = ["g++", "-O1", "-std=c++17", "-pthread", "-I", cuda_inc, "-I",
           os.path.join(root, "include"), "-I", os.path.join(root, "sih26_b200", "csrc"),
           os.path.join(here, "certificate_check.cpp"),
           os.path.join(root, "sih26_b200", "csrc", "pdhg_host.cpp"), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:  # the host source may want the CUDA runtime's symbols at link time
        r = subprocess.run(cmd + ["-L/usr/local/cuda/lib64", "-lcudart"], capture_output=True,
                           text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return exe


def _run_checker(exe, tmp_path, cases):
    """cases: (name, kind, dense rows, row_lower, row_upper, cost, col_lower, col_upper,
    vector); returns {name: [verdicts]}."""
    import subprocess

    lines = []
    for name, kind, rows, rl, ru, cost, cl, cu, vec in cases:
        toks = [name, kind, str(len(rl)), str(len(cost))]
        toks += [repr(float(v)) for row in rows for v in row]
        toks += [repr(float(v)) for v in (*rl, *ru, *cost, *cl, *cu, *vec)]
        lines.append(" ".join(toks))
    path = tmp_path / "cases.txt"
    path.write_text("\n".join(lines) + "\n")
    out = subprocess.run([str(exe), str(path)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    return {line.split()[0]: line.split()[1:] for line in out.stdout.splitlines()}


def test_library_checkers_give_the_reference_known_answers(cert_checker, tmp_path):
    """The library's own farkas_holds / ray_holds (pdhg_host.cpp), through
    tests/certificate_check.cpp compiled against the library's host source."""
    got = _run_checker(cert_checker, tmp_path, [c[:9] for c in KNOWN_ANSWERS])
    assert got == {c[0]: ["1" if c[9] else "0"] for c in KNOWN_ANSWERS}


def _dense(lp):
    a = np.zeros((lp.num_rows, lp.num_cols))
    for j in range(lp.num_cols):
        for k in range(lp.col_starts[j], lp.col_starts[j + 1]):
            a[lp.row_indices[k], j] = lp.values[k]
    return a.tolist()


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_ray_repair_recovers_a_planted_ray_and_never_makes_a_proof(cert_checker, tmp_path,
                                                                   seed):
    """repair_ray (pdhg_host.cpp) on primal-ray candidates like the ones PDHG iterates leave
    behind: the planted ray of an unbounded LP (lpgen.make_unbounded) passes as it is and after
    the repair; with the two ray columns moving 2e-6 apart and 1e-7 noise on every bounded
    column it fails as it is (rows and bounds move) and passes once repaired; a negated
    candidate and a random direction stay rejected, since the repaired vector must still pass
    the reference's rules (certificate.cpp:121-218)."""
    rng = np.random.default_rng(seed)
    lp = _unbounded(seed)
    n = lp.num_cols
    noisy = lp.ray_star.copy()
    noisy[-1] += 2e-6
    noisy[:-2] += 1e-7 * rng.standard_normal(n - 2)
    vectors = {"exact": lp.ray_star, "noisy": noisy, "negated": -noisy,
               "random": rng.standard_normal(n)}
    rows = _dense(lp)
    cases = [(name, "P", rows, lp.row_lower, lp.row_upper, lp.cost, lp.col_lower, lp.col_upper,
              vec) for name, vec in vectors.items()]
    got = _run_checker(cert_checker, tmp_path, cases)
    assert got == {"exact": ["1", "1"], "noisy": ["0", "1"], "negated": ["0", "0"],
                   "random": ["0", "0"]}, got
    # the numpy restatement agrees on the candidates as they are
    for name, vec in vectors.items():
        assert ray_numpy(lp, vec)[0] == (got[name][0] == "1"), name
