"""The autotuner's cache file on the CPU (sih26_b200/csrc/pdhg_host.cpp: the single-LP
schedules and the served chunk length): stored picks read back, the last line of a key wins,
keys match whole, and damaged lines are ignored, through tests/cache_check.cpp compiled
against the library's host source. The GPU tests measure and reuse real picks
(tests/test_gpu_autotune.py, tests/test_gpu_server_autotune.py)."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CUDA_INC = "/usr/local/cuda/include"


def test_cache_file_reads_back_and_ignores_damage(tmp_path):
    if shutil.which("g++") is None or not os.path.isdir(CUDA_INC):
        pytest.skip("no C++ compiler or CUDA headers")
    exe = tmp_path / "cache_check"
    cmd = ["g++", "-O1", "-std=c++17", "-pthread", "-I", CUDA_INC, "-I",
           os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "sih26_b200", "csrc"),
           os.path.join(HERE, "cache_check.cpp"),
           os.path.join(ROOT, "sih26_b200", "csrc", "pdhg_host.cpp"), "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:  # the host source may want the CUDA runtime's symbols at link time
        r = subprocess.run(cmd + ["-L/usr/local/cuda/lib64", "-lcudart"], capture_output=True,
                           text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    scratch = tmp_path / "scratch"
    scratch.mkdir()
    out = subprocess.run([str(exe), str(scratch)], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr
    assert (scratch / "a" / "b" / "c" / "autotune.tsv").exists()
