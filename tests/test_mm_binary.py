"""The reference's binary .mm matrix file (abhsf_read_mm / abhsf_write_mm,
host code of the library): the byte layout utils/mtx2mm/mtx2mm.cpp:102-135
writes, built here with struct from that layout, and reading it back gives
what the reference's text reader gave for the same matrix
(tests/golden/mtx_ref.npz)."""
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN
from abhsf_b200 import capi
from abhsf_b200 import matrix as mx

REF = np.load(os.path.join(GOLDEN, "mtx_ref.npz"))
NAMES = sorted({k.split("__")[0] for k in REF.files})


def mtx2mm_bytes(m, n, rows, cols, vals, type_code, flag):
    """The bytes mtx2mm.cpp:102-135 writes: u64 m, n, nnz, type, hermit; u32
    rows; u32 cols; f64 values (real only)."""
    out = struct.pack("<5Q", m, n, len(rows), type_code, flag)
    out += np.asarray(rows, "<u4").tobytes() + np.asarray(cols, "<u4").tobytes()
    if type_code == 2:
        out += np.asarray(vals, "<f8").tobytes()
    return out


@pytest.mark.parametrize("name", NAMES)
def test_mtx2mm_round_trip_is_the_reference_reader(tmp_path, name):
    src = os.path.join(GOLDEN, "mtx", name + ".mtx")
    dst = str(tmp_path / (name + ".mm"))
    mx.mtx2mm(src, dst)
    rows, cols, vals, m, n, info = mx.read_mm(dst)
    assert [m, n] == REF[name + "__shape"].tolist()
    np.testing.assert_array_equal(rows, REF[name + "__rows"])
    np.testing.assert_array_equal(cols, REF[name + "__cols"])
    np.testing.assert_array_equal(vals.view(np.uint64), REF[name + "__vals"].view(np.uint64))
    assert info == mx.read_mtx(src)[5]
    # and the bytes are the mtx2mm layout
    binary = info["matrix_type"] == "binary"
    flag = {"general": 0, "symmetric": 1, "hermitian": 2, "skew": 3}[info["symmetry"]]
    want = mtx2mm_bytes(m, n, rows, cols, vals, 0 if binary else 2, flag)
    assert open(dst, "rb").read() == want


def test_reference_written_file_with_zeros_reads_like_the_text_reader(tmp_path):
    """mtx2mm keeps explicit zeros (it writes every element it read) and
    writes its symmetry flag as a bool: read back, the zeros are dropped as
    read_mtx_real_or_binary drops them and a flag of 1 is symmetric."""
    rows, cols = [0, 1, 2, 2], [0, 0, 1, 2]
    vals = [2.5, 0.0, -1.0, 0.0]
    p = tmp_path / "z.mm"
    p.write_bytes(mtx2mm_bytes(3, 3, rows, cols, vals, 2, 1))
    r, c, v, m, n, info = mx.read_mm(str(p))
    np.testing.assert_array_equal(r, [0, 2])
    np.testing.assert_array_equal(c, [0, 1])
    np.testing.assert_array_equal(v, [2.5, -1.0])
    assert (m, n) == (3, 3)
    assert info == {"matrix_type": "real", "symmetry": "symmetric", "stored_triangle": "lower"}
    t = tmp_path / "z.mtx"
    t.write_text("%%MatrixMarket matrix coordinate real symmetric\n3 3 4\n1 1 2.5\n2 1 0\n3 2 -1\n3 3 0\n")
    text = mx.read_mtx(str(t))
    for a, b in zip(text[:3], (r, c, v)):
        np.testing.assert_array_equal(a, b)
    assert text[3:] == (m, n, info)


def test_pattern_and_large_round_trip(tmp_path):
    rng = np.random.default_rng(11)
    m, n, k = 70000, 50000, 300000
    rows = rng.integers(0, m, k)
    cols = rng.integers(0, n, k)
    vals = rng.standard_normal(k)
    p = str(tmp_path / "a.mm")
    mx.write_mm(p, rows, cols, vals, m, n)
    r, c, v, mm, nn, info = mx.read_mm(p)
    np.testing.assert_array_equal(r, rows)
    np.testing.assert_array_equal(c, cols)
    np.testing.assert_array_equal(v.view(np.uint64), vals.view(np.uint64))
    assert (mm, nn, info["matrix_type"], info["symmetry"]) == (m, n, "real", "general")
    assert os.path.getsize(p) == 40 + 16 * k
    mx.write_mm(p, rows, cols, None, m, n, matrix_type="binary")
    r, c, v, _, _, info = mx.read_mm(p)
    np.testing.assert_array_equal(r, rows)
    assert info["matrix_type"] == "binary" and np.all(v == 1.0)
    assert os.path.getsize(p) == 40 + 8 * k
    mx.write_mm(p, [], [], [], 5, 4)  # no elements
    r, c, v, mm, nn, _ = mx.read_mm(p)
    assert r.size == c.size == v.size == 0 and (mm, nn) == (5, 4)


@pytest.mark.parametrize("payload,exc", [
    (mtx2mm_bytes(2, 2, [0], [0], [1.0], 1, 0), capi.Unsupported),          # integer
    (mtx2mm_bytes(2, 2, [0], [0], [1.0], 3, 0), capi.Unsupported),          # complex
    (mtx2mm_bytes(2, 2, [0], [0], [1.0], 7, 0), capi.InvalidValue),         # no such type
    (mtx2mm_bytes(2, 2, [0], [0], [1.0], 2, 9), capi.InvalidValue),         # no such symmetry
    (mtx2mm_bytes(2, 2, [2], [0], [1.0], 2, 0), capi.IndexOutOfRange),      # row past m
    (mtx2mm_bytes(2, 2, [0], [5], [1.0], 2, 0), capi.IndexOutOfRange),      # col past n
    (mtx2mm_bytes(3, 3, [1, 0], [0, 1], [1.0, 1.0], 2, 1), capi.InvalidValue),  # both triangles
    (mtx2mm_bytes(2, 2, [0], [0], [1.0], 2, 0)[:-4], capi.InvalidValue),    # truncated
    (mtx2mm_bytes(2, 2, [0], [0], [1.0], 2, 0) + b"\0", capi.InvalidValue),  # trailing bytes
    (struct.pack("<5Q", 2, 2, 1 << 62, 2, 0), capi.InvalidValue),           # nnz past the file
    (struct.pack("<5Q", 0, 2, 0, 2, 0), capi.InvalidValue),                 # m = 0
    (b"\0" * 12, capi.InvalidValue),                                        # no header
])
def test_read_errors(tmp_path, payload, exc):
    p = tmp_path / "bad.mm"
    p.write_bytes(payload)
    with pytest.raises(exc):
        mx.read_mm(str(p))


def test_write_errors(tmp_path):
    p = str(tmp_path / "w.mm")
    with pytest.raises(capi.IndexOutOfRange):
        mx.write_mm(p, [0, 3], [0, 0], [1.0, 1.0], 3, 3)
    with pytest.raises(capi.InvalidValue):
        mx.write_mm(p, [0], [0], [1.0], (1 << 32) + 1, 3)  # u32 indices reach 2^32 rows at most
    with pytest.raises(capi.InvalidValue):
        mx.write_mm(p, [0], [0], [1.0], 3, 3, symmetry="diagonal")
    with pytest.raises(capi.InvalidValue):
        mx.read_mm(str(tmp_path / "missing.mm"))
