"""The host work partition (sih26_b200/csrc/pdhg_host.cpp: partition) on the CPU.

Every kernel of the single-LP and batched engines walks this partition: stream items or slices
of short rows, grouped rows, segments of long rows, assigned to blocks. tests/partition_check.cpp
is compiled here against the library's host source and checks, for row-length distributions of
the benched families and edge cases, that every row is owned exactly once, that segments tile
their rows, that the per-block index arrays are consistent, and that slices are in bounds and
disjoint. It also pins the bound the batched pool sizing relies on: with rows sorted longest
first (as the engines sort them), the slice arrays hold at most the sliced rows' nonzeros plus
32 x 32 entries of padding.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from sih26_b200 import lpgen

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA_INC = "/usr/local/cuda/include"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.isdir(CUDA_INC):
        pytest.skip("no C++ compiler or CUDA headers")
    exe = tmp_path_factory.mktemp("part") / "partition_check"
    cmd = ["g++", "-O1", "-std=c++17", "-pthread", "-I", CUDA_INC, "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "sih26_b200", "csrc"), os.path.join(HERE, "partition_check.cpp"),
           os.path.join(ROOT, "sih26_b200", "csrc", "pdhg_host.cpp"), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:  # the host source may want the CUDA runtime's symbols at link time
        r = subprocess.run(cmd + ["-L/usr/local/cuda/lib64", "-lcudart"], capture_output=True,
                           text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return exe


def _lengths():
    lp = lpgen.powerlaw_planted(m=20_000, n=50_000, seed=4)
    rows = np.bincount(lp.row_indices, minlength=lp.num_rows)
    cols = np.diff(lp.col_starts)
    mixed = np.array([5000, 1200, 600, 513, 512, 511, 300, 100, 64, 33, 32, 31, 17, 16, 9, 2, 1, 1,
                      0, 0] + [3] * 70 + [40] * 9)
    rng = np.random.default_rng(1)
    return {"powerlaw rows": rows, "powerlaw columns": cols, "mixed": mixed,
            "uniform 0-40": rng.integers(0, 41, 3000), "one row": np.array([7]),
            "no rows": np.array([], dtype=np.int64), "one long row": np.array([4097])}


@pytest.mark.parametrize("sliced", [True, False])
@pytest.mark.parametrize("G,sched", [(296, (32, 16)), (296, (16, 8)), (8, (32, 32)), (1, (8, 16))])
def test_partition_invariants(checker, tmp_path, sliced, G, sched):
    for name, lens in _lengths().items():
        lens = np.sort(np.asarray(lens, dtype=np.int32))[::-1]  # longest first, as the engines
        path = tmp_path / "lens.bin"
        lens.astype(np.int32).tofile(path)
        r = subprocess.run([str(checker), str(path), str(G), str(sched[0]), str(sched[1]),
                            str(int(sliced))], capture_output=True, text=True)
        out = r.stdout.strip()
        assert r.returncode == 0 and out.startswith("ok"), (name, G, sched, sliced, out, r.stderr)
        f = dict(zip(out.split()[1::2], map(int, out.split()[2::2])))
        assert f["rows"] == len(lens)
        if sliced:
            assert f["sell"] <= f["slice_nnz"] + 32 * 32, (name, f)
