"""The C-ABI library: it loads, exports every symbol include/*.h declares, mirrors the
reference's option names and defaults, and rejects bad input before touching a GPU."""
import ctypes as C
import dataclasses
import math
import os
import re

import numpy as np
import pytest

from sih26_b200 import build, lpgen
from sih26_b200 import pdhg as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build_library()
    return P.load_library()


def _declared_functions():
    names = []
    inc = os.path.join(ROOT, "include")
    for f in sorted(os.listdir(inc)):
        if f.endswith(".h"):
            text = open(os.path.join(inc, f)).read()
            names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\**\s+\**(sankhya_[a-z_0-9]+)\s*\(",
                                text, flags=re.M)
    return names


def test_library_exports_every_declared_symbol(lib):
    declared = _declared_functions()
    assert set(P.EXPORTED_SYMBOLS) <= set(declared)
    for name in declared:
        assert hasattr(lib, name), name


def test_default_params_mirror_reference_option_defaults(lib):
    prm = P._Params()
    lib.sankhya_pdhg_gpu_default_params(C.byref(prm))
    # src/util/options.cpp: pdhg_tolerance = kPdhgLoose 1e-4, iteration_limit -1, time_limit
    # no limit, pdhg_restart true, pdhg_stop_at_request false, random_seed 0
    assert prm.tolerance == 1e-4
    assert prm.iteration_limit == -1
    assert math.isinf(prm.time_limit)
    assert prm.restart == 1 and prm.stop_at_request == 0 and prm.random_seed == 0
    opts = P.Options()
    assert opts.get("pdhg_tolerance") == prm.tolerance
    assert opts.get("iteration_limit") == prm.iteration_limit


def test_options_parse_like_the_cli():
    opts = P.Options()
    opts.set_from_string("pdhg_tolerance=1e-6")
    opts.set_from_string("pdhg_stop_at_request=true")
    opts.set_from_string("pdhg_precision=mixed")
    assert opts.get("pdhg_tolerance") == 1e-6
    assert opts.get("pdhg_stop_at_request") is True
    with pytest.raises(KeyError):
        opts.set("no_such_option", 1)
    with pytest.raises(ValueError):
        opts.set("pdhg_precision", "fp16")


def _tiny():
    return lpgen.from_dense([[1, 1]], [2], [math.inf], [1, 1])


def test_malformed_matrix_is_an_argument_error(lib):
    lp = _tiny()
    lp.row_indices = np.array([0, 5], dtype=np.int32)  # row 5 of a 1-row matrix
    with pytest.raises(P.GpuError) as e:
        P.solve_pdhg(lp)
    assert e.value.code == 10 and "out of range" in str(e.value)


def test_col_starts_are_checked_before_any_column_is_read(lib):
    # col_starts rises past num_nonzeros and then falls back to it: reading column 0's entries
    # first would run past the arrays, so the decrease must be found before any entry is read
    lp = lpgen.from_dense([[1, 1, 1]], [3], [math.inf], [1, 1, 1])
    lp.col_starts = np.array([0, 1000, 1001, 3], dtype=np.int32)
    with pytest.raises(P.GpuError) as e:
        P.solve_pdhg(lp)
    assert e.value.code == 10 and "col_starts decreases at column 2" in str(e.value)


def test_the_first_bad_column_is_reported_when_the_checks_run_in_parallel(lib):
    # 1M nonzeros: the entry checks run in several column ranges at once; the message must name
    # the first bad column in column order, as one pass would
    lp = lpgen.uniform_planted(40000, 100000, 10, seed=3)
    ri = lp.row_indices.copy()
    ri[lp.col_starts[90000]] = lp.num_rows  # out of range, late
    ri[lp.col_starts[20001] + 3] = -1       # out of range, earlier
    bad = dataclasses.replace(lp, row_indices=ri)
    with pytest.raises(P.GpuError) as e:
        P.solve_pdhg(bad)
    assert e.value.code == 10 and "in column 20001" in str(e.value)
    vals = lp.values.copy()
    vals[lp.col_starts[99000]] = math.inf
    vals[lp.col_starts[5000] + 1] = math.nan
    s = P.solve_pdhg(dataclasses.replace(lp, values=vals))
    row = int(lp.row_indices[lp.col_starts[5000] + 1])
    assert s.status == "model_error" and f"matrix entry ({row}, 5000) is nan" in s.message


def test_unsorted_column_is_an_argument_error(lib):
    lp = lpgen.from_dense([[1, 0], [1, 1]], [1, 1], [1, 1], [1, 1])
    lp.row_indices = lp.row_indices[[1, 0, 2]].copy()
    with pytest.raises(P.GpuError) as e:
        P.solve_pdhg(lp)
    assert e.value.code == 10


def test_model_errors_come_back_as_a_status(lib):
    # Model::validate (src/core/model.cpp:188-206) wording; pdhg.cpp:273-278 returns it
    lp = _tiny()
    lp.col_lower = np.array([3.0, 0.0])
    lp.col_upper = np.array([1.0, math.inf])
    s = P.solve_pdhg(lp)
    assert s.status == "model_error"
    assert "column 0 has lower bound 3 above upper bound 1" in s.message
    lp = _tiny()
    lp.values = np.array([math.nan, 1.0])
    s = P.solve_pdhg(lp)
    assert s.status == "model_error" and "not a usable coefficient" in s.message


def test_no_cpu_fallback_without_a_gpu(lib):
    if P.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(P.GpuError) as e:
        P.solve_pdhg(_tiny())
    assert e.value.code == 2


@pytest.mark.skipif(not any(os.access(os.path.join(d, "gcc"), os.X_OK)
                            for d in os.environ.get("PATH", "").split(os.pathsep)),
                    reason="no C compiler")
def test_python_mirrors_match_the_header_layout(tmp_path):
    """Every ctypes mirror in sih26_b200/pdhg.py has the size and field offsets the C compiler
    gives the header's struct (a field added to one side only would shift the others)."""
    import subprocess

    pairs = [("sankhya_pdhg_problem", P._Problem), ("sankhya_pdhg_params", P._Params),
             ("sankhya_pdhg_residuals", P._Residuals), ("sankhya_pdhg_quality", P._Quality),
             ("sankhya_pdhg_result", P._Result), ("sankhya_pdhg_server_config", P._ServerConfig),
             ("sankhya_pdhg_server_stats", P._ServerStats), ("sankhya_qp_hessian", P._Hessian)]
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "sankhya_pdhg_gpu.h"',
             "int main(void) {"]
    for cname, py in pairs:
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        cname, key, val = line.split()
        got[(cname, key)] = int(val)
    for cname, py in pairs:
        assert got[(cname, "size")] == C.sizeof(py), cname
        for field, _ in py._fields_:
            assert got[(cname, field)] == getattr(py, field).offset, (cname, field)


def test_server_defaults_and_stats_arguments(lib):
    """The served engine's defaults (chunk length autotuned, 8-block clusters from 16,384
    nonzeros, no solo routing) and the stats entry point's argument check, without a GPU."""
    P._bind_server(lib)
    cfg = P._ServerConfig()
    lib.sankhya_pdhg_server_default_config(C.byref(cfg))
    assert cfg.chunk_attempts == -1
    assert cfg.cluster_min_nnz == 16384 and cfg.clusters == 0 and cfg.solo_min_nnz == 0
    assert cfg.max_active == 4096 and abs(cfg.memory_fraction - 0.8) < 1e-12
    st = P._ServerStats()
    assert lib.sankhya_pdhg_server_get_stats(None, C.byref(st)) == 10
    assert "must not be NULL" in lib.sankhya_pdhg_gpu_last_error().decode()


def _malformed():
    """LPs that break one rule of Model::validate each (src/core/model.cpp:125-210), with the
    formatting edge cases of its messages, and two that break several (the first rule wins)."""
    def base():
        return lpgen.uniform_planted(6, 10, 3, seed=1)

    def edit(**arrays):
        lp = base()
        for name, (index, value) in arrays.items():
            a = np.array(getattr(lp, name), dtype=np.float64)
            a[index] = value
            setattr(lp, name, a)
        return lp

    cases = [
        ("nan_entry", edit(values=(4, math.nan))),
        ("neg_nan_entry", edit(values=(4, -math.nan))),
        ("inf_entry", edit(values=(0, math.inf))),
        ("neg_inf_entry", edit(values=(7, -math.inf))),
        ("nan_col_lower", edit(col_lower=(3, math.nan))),
        ("nan_col_upper", edit(col_upper=(9, math.nan))),
        ("crossed_col", edit(col_lower=(2, 3.0), col_upper=(2, 1.0))),
        ("crossed_col_wide", edit(col_lower=(5, 1e300), col_upper=(5, 2.5e-7))),
        ("crossed_col_inf", edit(col_lower=(1, math.inf), col_upper=(1, -math.inf))),
        ("nan_cost", edit(cost=(8, math.nan))),
        ("nan_row_bound", edit(row_upper=(2, math.nan))),
        ("crossed_row", edit(row_lower=(4, 0.1), row_upper=(4, -1234567.0))),
        ("nan_offset", base()),
        ("entry_before_bounds", edit(values=(12, math.nan), col_lower=(0, math.nan))),
        ("col_before_row", edit(cost=(9, math.nan), row_lower=(0, math.nan))),
    ]
    cases[12][1].objective_offset = math.nan
    big = lpgen.uniform_planted(20000, 100000, 10, seed=2)  # ~1M nonzeros: parallel scan
    v = np.array(big.values)
    v[len(v) - 5] = math.inf
    v[len(v) // 2] = math.nan
    big.values = v
    cases.append(("first_of_two_entries", big))
    return cases


@pytest.mark.parametrize("name,lp", _malformed(), ids=[c[0] for c in _malformed()])
def test_model_error_text_is_the_reference_validate_text(lib, name, lp):
    """The MODEL_ERROR message is Model::validate's text, as solve_pdhg reports it
    (src/pdhg/pdhg.cpp:273-278), character for character, checked on the host before any GPU
    work (so it runs here)."""
    import oracle

    if not oracle.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")
    want = oracle.ref_validate(lp)
    assert want, name
    s = P.solve_pdhg(lp)
    assert s.status == "model_error", (name, s.status, s.message)
    assert s.message == want, (name, s.message, want)
