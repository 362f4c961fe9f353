"""The request wire format (sankhya_pdhg_wire_*): host-only functions of the library, so these
run without a GPU. Round trips, the layout decoded independently with numpy, and the inputs
the reader must turn down."""
import math
import struct

import numpy as np
import pytest

from sih26_b200 import lpgen
from sih26_b200 import pdhg as P


def _lps():
    yield lpgen.uniform_planted(60, 150, 4, seed=1)
    yield lpgen.from_dense([[1, 0], [0, 2], [3, 2]], [-math.inf] * 3, [4, 12, 18], [3, 5],
                           maximize=True, objective_offset=2.5)
    yield lpgen.from_dense([[1]], [2], [6], [1])  # odd sizes: padding of the int32 arrays


@pytest.mark.parametrize("lp", list(_lps()), ids=["uniform", "maximise", "one-by-one"])
def test_round_trip_keeps_every_bit(lp):
    buf = P.to_wire(lp)
    back = P.from_wire(buf)
    assert (back.num_rows, back.num_cols, back.maximize) == (lp.num_rows, lp.num_cols, lp.maximize)
    assert back.objective_offset == lp.objective_offset
    for f in ("col_starts", "row_indices", "values", "cost", "col_lower", "col_upper",
              "row_lower", "row_upper"):
        a, b = np.asarray(getattr(lp, f)), getattr(back, f)
        assert a.shape == b.shape and np.array_equal(a, b, equal_nan=True), f


def test_layout_decoded_with_numpy():
    lp = lpgen.uniform_planted(7, 9, 3, seed=4)
    buf = P.to_wire(lp).tobytes()
    assert buf[:8] == b"SKPDHG01"
    m, n, nnz, flags = struct.unpack_from("<4i", buf, 8)
    assert (m, n, nnz, flags) == (7, 9, lp.num_nonzeros, 0)
    at = 32

    def take(count, dtype):
        nonlocal at
        a = np.frombuffer(buf, dtype=dtype, count=count, offset=at)
        at = (at + a.nbytes + 7) // 8 * 8
        return a

    assert np.array_equal(take(n + 1, "<i4"), lp.col_starts)
    assert np.array_equal(take(nnz, "<i4"), lp.row_indices)
    assert np.array_equal(take(nnz, "<f8"), lp.values)
    for f in ("cost", "col_lower", "col_upper"):
        assert np.array_equal(take(n, "<f8"), getattr(lp, f))
    for f in ("row_lower", "row_upper"):
        assert np.array_equal(take(m, "<f8"), getattr(lp, f))
    assert at == len(buf)


def test_reader_turns_down_bad_buffers():
    good = P.to_wire(lpgen.uniform_planted(20, 40, 3, seed=2)).tobytes()
    for bad, why in ((b"NOTWIRE!" + good[8:], "magic"), (good[:len(good) - 8], "truncated"),
                     (good[:16], "header")):
        with pytest.raises(P.GpuError) as e:
            P.from_wire(bad)
        assert e.value.code == 10, why
    # a row index out of range is caught by the structural check
    corrupt = bytearray(good)
    m, n, nnz, _ = struct.unpack_from("<4i", good, 8)
    ri_at = 32 + ((n + 1) * 4 + 7) // 8 * 8
    struct.pack_into("<i", corrupt, ri_at, m + 5)
    with pytest.raises(P.GpuError):
        P.from_wire(bytes(corrupt))
