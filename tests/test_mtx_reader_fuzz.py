"""Matrix Market ingest (abhsf_read_mtx) against the reference's own reader,
read_mtx_real_or_binary (include/abhsf/utils/matrix_market_reader.h:146-200),
on generated files: random sizes, real or pattern, general or one triangle
of a symmetric matrix, values in several printed forms (17 and 7 significant
digits, integers, zeros of both signs, subnormals, huge and tiny exponents),
tabs and runs of spaces, CRLF line ends, comment lines.  The reference's
reader is compiled from its sources into oracle/_ref/libref_mtx.so (the
checker); without it the test is skipped."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from abhsf_b200 import capi
from abhsf_b200 import matrix as mx

hyp = pytest.importorskip("hypothesis")
st = pytest.importorskip("hypothesis.strategies")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_mtx.so")
pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="reference reader not built (make -C oracle ref)")


def ref_read(path: str):
    lib = C.CDLL(LIB)
    f = lib.ref_mtx_read
    f.restype = C.c_long
    cap = 1 << 16
    m, n = C.c_long(), C.c_long()
    rows, cols, vals = np.zeros(cap, np.int64), np.zeros(cap, np.int64), np.zeros(cap, np.float64)
    k = f(os.fsencode(path), C.byref(m), C.byref(n), C.c_long(cap), rows.ctypes.data_as(C.c_void_p),
          cols.ctypes.data_as(C.c_void_p), vals.ctypes.data_as(C.c_void_p))
    assert k != -2
    if k < 0:
        return None
    return rows[:k], cols[:k], vals[:k], m.value, n.value


def value_text(draw_kind: int, v: float) -> str:
    if draw_kind == 0:
        return f"{v:.17g}"
    if draw_kind == 1:
        return f"{v:.6e}"
    if draw_kind == 2:
        return str(int(round(v)))
    if draw_kind == 3:
        return ("-0.0", "0", "0.000e+00", "+0")[int(abs(v) * 1000) % 4]
    if draw_kind == 4:
        return f"{v * 1e-310:.17g}"  # subnormal
    return f"{v * 10.0 ** (int(abs(v) * 1e6) % 600 - 300):.15g}"  # exponents from -300 to 299


@st.composite
def mtx_files(draw):
    m = draw(st.integers(1, 40))
    n = draw(st.integers(1, 40))
    pattern = draw(st.booleans())
    symmetric = draw(st.booleans()) and m == n
    lower = draw(st.booleans())
    k = draw(st.integers(0, 60))
    ents = []
    for _ in range(k):
        i = draw(st.integers(1, m))
        j = draw(st.integers(1, n))
        if symmetric and ((i < j) if lower else (i > j)):
            i, j = j, i
        kind = draw(st.integers(0, 5))
        v = draw(st.floats(-1e3, 1e3, allow_nan=False, allow_infinity=False))
        ents.append((i, j, value_text(kind, v)))
    sep = draw(st.sampled_from([" ", "\t", "  ", " \t "]))
    eol = draw(st.sampled_from(["\n", "\r\n"]))
    trailing = draw(st.sampled_from(["", " ", "\t"]))
    comments = draw(st.integers(0, 3))
    field = "pattern" if pattern else "real"
    sym = "symmetric" if symmetric else "general"
    lines = [f"%%MatrixMarket matrix coordinate {field} {sym}"]
    lines += ["% comment " + "x" * c for c in range(comments)]
    lines.append(f"{m} {n} {k}")
    for i, j, t in ents:
        lines.append(sep.join([str(i), str(j)] + ([] if pattern else [t])) + trailing)
    return eol.join(lines) + eol


@hyp.settings(max_examples=150, deadline=None, derandomize=True)
@hyp.given(text=mtx_files(), threads=st.sampled_from([1, 3]))
def test_generated_files_read_like_the_reference_reader(text, threads):
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "a.mtx")
        with open(p, "w", newline="") as f:
            f.write(text)
        want = ref_read(p)
        if want is None:  # the reference's reader threw: ours raises as well
            with pytest.raises(capi.AbhsfError):
                mx.read_mtx(p, threads)
            return
        rows, cols, vals, m, n, _ = mx.read_mtx(p, threads)
        assert (m, n) == (want[3], want[4])
        np.testing.assert_array_equal(rows, want[0])
        np.testing.assert_array_equal(cols, want[1])
        np.testing.assert_array_equal(vals.view(np.uint64), want[2].view(np.uint64))
        # and through the binary layout
        mm = os.path.join(d, "a.mm")
        mx.mtx2mm(p, mm)
        r2, c2, v2, m2, n2, _ = mx.read_mm(mm)
        assert (m2, n2) == (m, n)
        np.testing.assert_array_equal(r2, rows)
        np.testing.assert_array_equal(c2, cols)
        np.testing.assert_array_equal(v2.view(np.uint64), vals.view(np.uint64))
