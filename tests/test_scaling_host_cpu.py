"""The library's host build_scaling (sih26_b200/csrc/pdhg_host.cpp) against the reference's
own build_scaling (src/la/scaling.cpp:111-158, compiled in oracle/_ref), bit for bit.

The host version prepares every LP of the batched and served engines and every single LP below
the device-preparation threshold, and the device version is tested against it on the GPU
(tests/test_gpu_prep.py); this pins the host version to the reference directly. It runs through
tests/scaling_check.cpp, compiled here against the library's host source, on LPs with every
bound and row kind, both senses (the min-space cost of a maximised LP is the negated cost, as
pdhg.cpp:287-291 forms it), block-angular long rows, and a 2M-nonzero power-law LP whose row
and column passes are split over several host threads. The norm estimate's random start
(uniform_draws) is pinned to the standard library's draws the same way, and the host layout
(permute: length-sorted CSR copies of A and A') is checked against the CSC it came from.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from cases import generated_cases
from sih26_b200 import lpgen
from test_quality_oracle import edge_lps

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA_INC = "/usr/local/cuda/include"
KEYS = ("row_scale", "col_scale", "values", "cost", "col_lower", "col_upper", "row_lower",
        "row_upper")


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.isdir(CUDA_INC):
        pytest.skip("no C++ compiler or CUDA headers")
    if not oracle.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    exe = tmp_path_factory.mktemp("scaling") / "scaling_check"
    cmd = ["g++", "-O2", "-std=c++17", "-pthread", "-I", CUDA_INC, "-I",
           os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "sih26_b200", "csrc"),
           os.path.join(HERE, "scaling_check.cpp"),
           os.path.join(ROOT, "sih26_b200", "csrc", "pdhg_host.cpp"), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:  # the host source may want the CUDA runtime's symbols at link time
        r = subprocess.run(cmd + ["-L/usr/local/cuda/lib64", "-lcudart"], capture_output=True,
                           text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return exe


def _lps():
    out = list(generated_cases()) + edge_lps()
    out.append(("block_angular", lpgen.block_angular_planted(blocks=6, block_rows=300,
                                                             block_cols=700, nnz_per_col=5,
                                                             linking_rows=20, seed=5)))
    out.append(("powerlaw_2M", lpgen.powerlaw_planted(m=80_000, n=200_000, seed=3)))
    return out


def _host_scaling(exe, tmp_path, lp, min_cost, ruiz):
    m, n, nnz = lp.num_rows, lp.num_cols, lp.num_nonzeros
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(src, "wb") as f:
        np.array([m, n, nnz, ruiz], dtype=np.int32).tofile(f)
        np.asarray(lp.col_starts, dtype=np.int32).tofile(f)
        np.asarray(lp.row_indices, dtype=np.int32).tofile(f)
        for a in (lp.values, min_cost, lp.col_lower, lp.col_upper, lp.row_lower, lp.row_upper):
            np.asarray(a, dtype=np.float64).tofile(f)
    r = subprocess.run([str(exe), str(src), str(dst)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
    flat = np.fromfile(dst, dtype=np.float64)
    sizes = (m, n, nnz, n, n, n, m, m)
    assert flat.size == sum(sizes)
    return dict(zip(KEYS, np.split(flat, np.cumsum(sizes)[:-1])))


@pytest.mark.parametrize("name,lp", _lps(), ids=[c[0] for c in _lps()])
def test_host_scaling_is_the_reference_scaling_bit_for_bit(checker, tmp_path, name, lp):
    min_cost = -np.asarray(lp.cost) if lp.maximize else np.asarray(lp.cost)
    for ruiz in (10, 0, 3):  # the solve's 10 rounds; none; a few
        mine = _host_scaling(checker, tmp_path, lp, min_cost, ruiz)
        ref = oracle.ref_scaling(lp, min_cost, ruiz)
        for k in KEYS:
            # equal bits: the same values, with infinities and their signs in the same places
            assert np.array_equal(mine[k].view(np.int64), ref[k].view(np.int64)), (name, ruiz, k)


def test_host_draws_are_the_standard_library_draws(tmp_path):
    """The library's uniform_draws, the norm estimate's random start (and the QP engine's), is
    std::mt19937 with std::uniform_real_distribution<double> bit for bit, across the
    generator's 624-word twist boundaries (tests/draws_check.cpp)."""
    if shutil.which("g++") is None or not os.path.isdir(CUDA_INC):
        pytest.skip("no C++ compiler or CUDA headers")
    exe = tmp_path / "draws_check"
    cmd = ["g++", "-O2", "-std=c++17", "-pthread", "-I", CUDA_INC, "-I",
           os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "sih26_b200", "csrc"),
           os.path.join(HERE, "draws_check.cpp"),
           os.path.join(ROOT, "sih26_b200", "csrc", "pdhg_host.cpp"), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        r = subprocess.run(cmd + ["-L/usr/local/cuda/lib64", "-lcudart"], capture_output=True,
                           text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout


@pytest.fixture(scope="module")
def permuter(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.isdir(CUDA_INC):
        pytest.skip("no C++ compiler or CUDA headers")
    exe = tmp_path_factory.mktemp("permute") / "permute_check"
    cmd = ["g++", "-O2", "-std=c++17", "-pthread", "-I", CUDA_INC, "-I",
           os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "sih26_b200", "csrc"),
           os.path.join(HERE, "permute_check.cpp"),
           os.path.join(ROOT, "sih26_b200", "csrc", "pdhg_host.cpp"), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        r = subprocess.run(cmd + ["-L/usr/local/cuda/lib64", "-lcudart"], capture_output=True,
                           text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return exe


def _sorted_by_count_stable(perm, counts):
    """perm lists every index once, by count descending, ties in index order."""
    assert np.array_equal(np.sort(perm), np.arange(len(counts)))
    want = np.lexsort((np.arange(len(counts)), -counts))
    return np.array_equal(perm, want)


@pytest.mark.parametrize("name,lp", _lps(), ids=[c[0] for c in _lps()])
def test_host_permutation_holds_the_matrix_in_both_orders(permuter, tmp_path, name, lp):
    """The library's permute (pdhg_host.cpp), which lays out every LP the batched engine and
    the host preparation run: rows of A and of A' in nonzero order, longest first and stable,
    and both CSR copies hold exactly the CSC's entries, their column indices pointing into the
    other permuted space."""
    m, n, nnz = lp.num_rows, lp.num_cols, lp.num_nonzeros
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    with open(src, "wb") as f:
        np.array([m, n, nnz, 0], dtype=np.int32).tofile(f)
        np.asarray(lp.col_starts, dtype=np.int32).tofile(f)
        np.asarray(lp.row_indices, dtype=np.int32).tofile(f)
        for a in (lp.values, lp.cost, lp.col_lower, lp.col_upper, lp.row_lower, lp.row_upper):
            np.asarray(a, dtype=np.float64).tofile(f)
    r = subprocess.run([str(permuter), str(src), str(dst)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
    raw = open(dst, "rb").read()
    ints = np.frombuffer(raw, dtype=np.int32, count=m + n + (m + 1) + nnz + (n + 1) + nnz)
    rest = np.frombuffer(raw, dtype=np.float64, offset=ints.nbytes)
    row_perm, col_perm, a_ptr, a_idx, at_ptr, at_idx = np.split(
        ints, np.cumsum([m, n, m + 1, nnz, n + 1]))
    a_val, at_val = rest[:nnz], rest[nnz:]
    assert rest.size == 2 * nnz
    cs = np.asarray(lp.col_starts, dtype=np.int64)
    ri = np.asarray(lp.row_indices, dtype=np.int64)
    cols = np.repeat(np.arange(n), np.diff(cs))
    assert _sorted_by_count_stable(row_perm, np.bincount(ri, minlength=m))
    assert _sorted_by_count_stable(col_perm, np.diff(cs))
    ref = np.lexsort((cols, ri))
    want = (ri[ref], cols[ref], np.asarray(lp.values)[ref])
    # A in permuted row order, indices into the permuted columns
    assert a_ptr[0] == 0 and a_ptr[-1] == nnz and np.all(np.diff(a_ptr) >= 0)
    ra = row_perm[np.repeat(np.arange(m), np.diff(a_ptr))]
    ca = col_perm[a_idx]
    o = np.lexsort((ca, ra))
    assert np.array_equal(ra[o], want[0]) and np.array_equal(ca[o], want[1])
    assert np.array_equal(a_val[o], want[2])
    # A' in permuted column order, indices into the permuted rows
    assert at_ptr[0] == 0 and at_ptr[-1] == nnz and np.all(np.diff(at_ptr) >= 0)
    ct = col_perm[np.repeat(np.arange(n), np.diff(at_ptr))]
    rt = row_perm[at_idx]
    o = np.lexsort((ct, rt))
    assert np.array_equal(rt[o], want[0]) and np.array_equal(ct[o], want[1])
    assert np.array_equal(at_val[o], want[2])
