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


def _no_gpu() -> bool:
    import torch
    return not torch.cuda.is_available()


@pytest.mark.skipif(not _no_gpu(), reason="host-side validation check for machines without a GPU")
@hyp.settings(max_examples=300, deadline=None, derandomize=True)
@hyp.given(block_size=st.sampled_from([-1, 0, 1, 8, 16, 48, 64, 256, 512, 1 << 30]),
           value_type=st.integers(-1, 4), allow_csr=st.integers(-1, 2), matrix_type=st.integers(-1, 4),
           forced=st.integers(-2, 5), on_dev=st.integers(0, 1), sum_order=st.integers(-1, 2),
           bits=st.sampled_from([-1, 0, 16, 32, 64, 1 << 40]), selector=st.integers(-1, 4),
           panel=st.integers(-2, 40), nnz=st.integers(-1, 5), m=st.integers(-1, 70), n=st.integers(-1, 70),
           null_rows=st.booleans())
def test_build_validation_never_crashes(block_size, value_type, allow_csr, matrix_type, forced, on_dev, sum_order,
                                        bits, selector, panel, nnz, m, n, null_rows):
    """abhsf_build with any options and sizes returns a status: invalid ones
    are refused on the host, and on this machine (no GPU) every valid call
    fails at the device with a status too.  on_dev is only ever set together
    with NULL pointers here, which the library refuses before any device
    work whenever nnz > 0."""
    import ctypes as C
    o = capi.BuildOpts()
    capi.lib.abhsf_build_opts_default(C.byref(o))
    o.block_size, o.value_type, o.allow_csr, o.matrix_type = block_size, value_type, allow_csr, matrix_type
    o.forced_scheme, o.inputs_on_device, o.sum_order = forced, on_dev, sum_order
    o.bits_per_value, o.selector, o.slice_tile_nnz = bits, selector, panel
    k = max(nnz, 0)
    rows = np.zeros(max(k, 1), np.int64)
    cols = np.arange(max(k, 1), dtype=np.int64)
    vals = np.ones(max(k, 1))
    use_null = null_rows or on_dev
    h = C.c_void_p()
    rc = capi.lib.abhsf_build(None if use_null else rows.ctypes.data, None if use_null else cols.ctypes.data,
                              None if use_null else vals.ctypes.data, nnz, m, n, C.byref(o), None, C.byref(h))
    if rc == 0:  # only on a GPU machine
        assert capi.lib.abhsf_release(h) == 0
    else:
        assert isinstance(capi.lib.abhsf_last_error_string(), (bytes, str))


@pytest.mark.parametrize("threads", [1, 4])
@pytest.mark.parametrize("entry", ["-1 2 4.5", "2 -3 1.0", "-0 1 1.0", "18446744073709551615 1 2.0"])
def test_mtx_reader_refuses_signed_and_wrapped_indices(entry, threads):
    """An index written with a sign, or one that only fits after wrapping,
    lies outside m x n: the reference's fscanf("%lu") reads "-1" as 2^64 - 1,
    which is not a row of a 3 x 3 matrix."""
    text = f"%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1.0\n{entry}\n"
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "a.mtx")
        with open(p, "w") as f:
            f.write(text)
        with pytest.raises(capi.AbhsfError) as e:
            mx.read_mtx(p, threads)
        assert e.value.status == capi.INDEX_OUT_OF_RANGE
