"""The reference-side adapter (integration/pdhg_gpu_adapter.cpp), compiled against the
reference's own headers and linked against the reference's own objects (oracle/_ref) and this
library, then run through tests/adapter_check.cpp on a Model built with the reference's API.

Three adapter calls run: the single LP, a batch of two LPs (answers carrying the quality block
the device measured) and a convex QP. Without a GPU each must hand back kNumericalError with
the library's reason, never a CPU answer (the boundary has no fallback); with one, the known
optima: -36 at (2, 6) for the LP of tests/unit/test_pdhg.cpp:642-648 under the name
"pdhg-gpu", and 1/26 - 17 at (36/13, 63/13) for the QP under "qp-gpu". The adapter reads
the GPU option rows only where the registry has them, so it runs against the reference's
registry as it stands (whose typed accessors abort on an unknown name).
"""
import os
import shutil
import subprocess
import sysconfig

import pytest

import oracle
from sih26_b200 import pdhg

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF = "/root/reference"
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libsankhya_ref.so")


def test_adapter_builds_against_the_reference_and_reports_without_fallback(tmp_path):
    if shutil.which("g++") is None or not os.path.isdir(os.path.join(REF, "include")):
        pytest.skip("needs g++ and the reference tree's headers")
    if not oracle.ref_available() or not os.path.exists(pdhg.LIBPATH):
        pytest.skip("needs the reference build (oracle/_ref) and the built library")
    fmt_inc = os.path.join(sysconfig.get_paths()["purelib"], "torch", "include")
    exe = tmp_path / "adapter_check"
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-Werror", "-DFMT_HEADER_ONLY",
           "-I", os.path.join(REF, "include"), "-I", os.path.join(REF, "src"),
           "-I", os.path.join(ROOT, "include"), "-I", fmt_inc,
           os.path.join(ROOT, "integration", "pdhg_gpu_adapter.cpp"),
           os.path.join(HERE, "adapter_check.cpp"), REF_SO, pdhg.LIBPATH,
           "-Wl,-rpath," + os.path.dirname(REF_SO),
           "-Wl,-rpath," + os.path.dirname(pdhg.LIBPATH),
           "-fopenmp", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    calls = {}
    for line in out.stdout.strip().splitlines():
        if not line.startswith("call="):
            continue
        head, message = line.split(" message=", 1)
        fields = dict(tok.split("=", 1) for tok in head.split())
        fields["message"] = message
        calls[fields["call"]] = fields
    assert set(calls) == {"lp", "batch0", "batch1", "qp"}, out.stdout
    for name, f in calls.items():
        engine = "qp" if name == "qp" else "pdhg"
        assert f["algorithm"] == f"{engine}-gpu", f
        if f["status"] == "numerical_error":
            assert f["message"].startswith(f"GPU {engine.upper()}: "), f
            assert "device" in f["message"] and int(f["iterations"]) == 0, f
        elif name == "qp":
            assert f["status"] == "optimal", f
            assert abs(float(f["objective"]) - (1 / 26 - 17)) <= 1e-6 * 17, f
        else:
            assert f["status"] == "optimal", f
            assert abs(float(f["objective"]) + 36.0) <= 1e-6 * 36, f
