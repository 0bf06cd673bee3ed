"""The binary LP request format (b2_lp_write / b2_lp_read): round trips and
the checks that reject malformed files, on CPU."""
import os
import struct

import numpy as np
import pytest

import b200pdlp as B
from conftest import load_fixture


def _same_lp(a, b):
    assert (a.m, a.n) == (b.m, b.n) and a.obj_offset == b.obj_offset
    # the file keeps A in CSR with each row's entries in their COO order
    order = np.argsort(a.row, kind="stable")
    np.testing.assert_array_equal(b.row, a.row[order])
    np.testing.assert_array_equal(b.col, a.col[order])
    np.testing.assert_array_equal(b.val, a.val[order])
    for f in ("c", "rL", "rU", "l", "u"):
        np.testing.assert_array_equal(getattr(b, f), getattr(a, f))


@pytest.mark.parametrize("name", ["afiro", "israel", "tiny_range"])
def test_round_trip_fixtures(tmp_path, name):
    U = B.RangedLP.like(load_fixture(name)[0])
    p = str(tmp_path / f"{name}.b2lp")
    B.write_lp(p, U)
    assert B.lp_file_dims(p) == (U.m, U.n, U.nnz)
    _same_lp(U, B.read_lp(p))


def test_round_trip_generated_and_infinite_bounds(tmp_path):
    lp = B.gen_transport(30, 40, 5)  # u = +inf
    p = str(tmp_path / "t.b2lp")
    B.write_lp(p, lp)
    back = B.read_lp(p)
    _same_lp(B.RangedLP.like(lp), back)
    assert np.all(np.isinf(back.u))


def test_empty_lp(tmp_path):
    lp = B.RangedLP(0, 0, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0), np.zeros(0), np.zeros(0),
                    np.zeros(0), np.zeros(0), np.zeros(0), 3.5)
    p = str(tmp_path / "e.b2lp")
    B.write_lp(p, lp)
    back = B.read_lp(p)
    assert (back.m, back.n, back.nnz, back.obj_offset) == (0, 0, 0, 3.5)


def _corrupt(path, offset, data):
    with open(path, "r+b") as f:
        f.seek(offset)
        f.write(data)


def test_malformed_files_are_rejected(tmp_path):
    U = B.RangedLP.like(load_fixture("afiro")[0])
    good = str(tmp_path / "good.b2lp")
    B.write_lp(good, U)
    raw = open(good, "rb").read()

    def check(blob, what):
        p = str(tmp_path / (what + ".b2lp"))
        with open(p, "wb") as f:
            f.write(blob)
        with pytest.raises(B.B2Error) as e:
            B.read_lp(p)
        assert e.value.code == B.B2_ERR_INVALID, what

    check(b"NOTANLP!" + raw[8:], "magic")
    check(raw[:-8], "truncated")
    check(raw + b"\0" * 8, "trailing")
    # a decreasing row pointer
    ptr0 = 32
    blob = bytearray(raw)
    blob[ptr0 + 8:ptr0 + 16] = struct.pack("<q", 10**6)
    check(bytes(blob), "row_ptr")
    # a column index out of range
    col0 = 32 + 8 * (U.m + 1)
    blob = bytearray(raw)
    blob[col0:col0 + 4] = struct.pack("<i", U.n + 3)
    check(bytes(blob), "col")
    with pytest.raises(B.B2Error):
        B.read_lp(str(tmp_path / "missing.b2lp"))
