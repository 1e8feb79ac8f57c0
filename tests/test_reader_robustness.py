"""The host readers on malformed input (generated): every call either
returns elements inside the declared m x n or raises the library's error;
none crashes, hangs or allocates from an unchecked header."""
import os
import struct
import tempfile

import numpy as np
import pytest

from abhsf_b200 import capi
from abhsf_b200 import matrix as mx

hyp = pytest.importorskip("hypothesis")
st = pytest.importorskip("hypothesis.strategies")


def _check(result, m_max=None):
    rows, cols, vals, m, n, info = result
    assert rows.size == cols.size == vals.size
    if rows.size:
        assert rows.min() >= 0 and rows.max() < m and cols.min() >= 0 and cols.max() < n
    assert info["matrix_type"] in ("real", "binary")


@hyp.settings(max_examples=300, deadline=None, derandomize=True)
@hyp.given(m=st.integers(0, 2 ** 40), n=st.integers(0, 2 ** 40), nnz=st.integers(0, 2 ** 63 - 1),
           typ=st.integers(0, 9), flag=st.integers(0, 9), body=st.binary(max_size=200),
           cut=st.integers(0, 40))
def test_mm_reader_on_arbitrary_files(m, n, nnz, typ, flag, body, cut):
    data = struct.pack("<5Q", m, n, nnz, typ, flag)[: 40 - cut if cut < 40 else 40] + body
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "a.mm")
        with open(p, "wb") as f:
            f.write(data)
        try:
            _check(mx.read_mm(p))
        except capi.AbhsfError:
            pass


@st.composite
def noisy_mtx(draw):
    m = draw(st.integers(1, 30))
    n = draw(st.integers(1, 30))
    k = draw(st.integers(0, 20))
    field = draw(st.sampled_from(["real", "pattern", "integer", "complex", "bogus"]))
    sym = draw(st.sampled_from(["general", "symmetric", "skew-symmetric", "hermitian", "other"]))
    lines = [draw(st.sampled_from([f"%%MatrixMarket matrix coordinate {field} {sym}",
                                   "%%MatrixMarket matrix array real general", "%%MatrixMarket", ""]))]
    lines.append(draw(st.sampled_from([f"{m} {n} {k}", f"{m} {n}", f"-{m} {n} {k}", "x y z", f"{m} {n} {k + 5}"])))
    for _ in range(k):
        i = draw(st.integers(-2, m + 2))
        j = draw(st.integers(-2, n + 2))
        v = draw(st.sampled_from(["1.5", "-0", "nan", "inf", "1e999", "abc", "", "0x1p3", "+2", "7 8"]))
        lines.append(draw(st.sampled_from([f"{i} {j} {v}", f"{i} {j}", f"{i}", "%c", "", f"{i}\t{j}\t{v}"])))
    return "\n".join(lines) + draw(st.sampled_from(["", "\n", "\r\n"]))


@hyp.settings(max_examples=300, deadline=None, derandomize=True)
@hyp.given(text=noisy_mtx(), threads=st.sampled_from([1, 4]))
def test_mtx_reader_on_noisy_files(text, threads):
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "a.mtx")
        with open(p, "w", newline="") as f:
            f.write(text)
        try:
            res = mx.read_mtx(p, threads)
        except capi.AbhsfError:
            return
        _check(res)
        # what was read also writes and reads back through the binary layout
        q = os.path.join(d, "a.mm")
        rows, cols, vals, m, n, info = res
        mx.write_mm(q, rows, cols, vals, m, n, info["matrix_type"], info["symmetry"])
        back = mx.read_mm(q)
        for a, b in zip(back[:3], res[:3]):
            np.testing.assert_array_equal(np.asarray(a).view(np.uint64) if a.dtype == np.float64 else a,
                                          np.asarray(b).view(np.uint64) if b.dtype == np.float64 else b)
