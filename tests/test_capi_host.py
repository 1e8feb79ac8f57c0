"""The C-ABI library on a machine without a GPU: it loads, exports every
function include/abhsf/*.h declares, computes the host-side cost model and mmf
lines exactly as the reference does, and rejects bad arguments before any
device work."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden_stats
from abhsf_b200 import capi
from abhsf_b200 import matrix as mx
from oracle import oracle


def test_library_exports_every_declared_symbol():
    names = capi.header_functions()
    assert len(names) >= 13
    for nm in names:
        assert hasattr(capi.lib, nm), nm
        assert nm in capi.PROTOTYPES, nm
    assert capi.lib.abhsf_abi_version() == 1


def test_struct_layouts():
    assert C.sizeof(capi.BuildOpts) == 56
    assert C.sizeof(capi.Stats) == 208


def test_cost_model_matches_oracle():
    for r in (2, 16, 64, 256):
        for s in (2, 16, 64, 256):
            for z in sorted({1, 2, 7, r * s // 3, r * s // 2, r * s - 1, r * s}):
                if z < 1:
                    continue
                for sch in range(4):
                    assert mx.block_scheme_bits(sch, r, s, z, 64) == oracle.block_bits(sch, r, s, z, 64)
                for binary in (False, True):
                    for allow in (False, True):
                        got = mx.block_select_scheme(r, s, z, 64, binary, allow)
                        want = oracle.select_scheme(r, s, z, 64, binary, allow)
                        assert capi.SCHEME_NAMES.index(got) == want, (r, s, z, binary, allow)


@pytest.mark.parametrize("name", sorted(golden_stats()))
def test_library_mmf_lines_match_reference(name):
    g = golden_stats()[name]
    m, n, _, nnz, _, mtype, _ = g["props"]
    for l1, l2 in zip(g["mmf_single"], g["mmf_double"]):
        r, s = l1[0], l1[1]
        hist = {int(z): c for z, c in g["bstats"][f"{r}x{s}"].items()}
        o1, o2 = mx.mmf_line(m, n, nnz, mtype, r, s, hist)
        assert o1 == l1[2:] and o2 == l2[2:], (r, s)


def test_build_rejects_bad_options_before_device_work():
    rows = np.array([0, 1], dtype=np.int64)
    cols = np.array([0, 1], dtype=np.int64)
    vals = np.array([1.0, 2.0])
    for kw, exc in (({"block_size": 48}, capi.InvalidValue), ({"block_size": 8}, capi.InvalidValue),
                    ({"block_size": 512}, capi.InvalidValue), ({"forced_scheme": 7}, capi.InvalidValue),
                    ({"matrix_type": "complex"}, capi.Unsupported),
                    ({"matrix_type": "binary", "forced_scheme": "dense"}, capi.InvalidValue)):
        with pytest.raises(exc):
            mx.AbhsfMatrix.from_elements(rows, cols, vals, 2, 2, **kw)
    with pytest.raises(capi.InvalidValue):
        mx.AbhsfMatrix.from_elements(rows, cols, vals, 0, 2)
    with pytest.raises(capi.InvalidValue):
        mx.AbhsfMatrix.from_elements(rows, cols, None, 2, 2)  # values required unless binary
    with pytest.raises(capi.InvalidValue):
        mx.AbhsfMatrix.from_elements(rows, cols[:1], vals, 2, 2)


def test_null_handle_and_error_string():
    st = capi.lib.abhsf_spmv(None, None, None, None)
    assert st == capi.INVALID_VALUE
    assert b"NULL" in capi.lib.abhsf_last_error_string()
    with pytest.raises(capi.InvalidValue):
        capi.check(st)
    assert capi.lib.abhsf_release(None) == capi.SUCCESS
    A = mx.AbhsfMatrix()
    with pytest.raises(capi.InvalidValue):
        A.spmv(np.zeros(1), np.zeros(1))


def test_block_histogram_argument_checks():
    with pytest.raises(capi.InvalidValue):
        mx.block_histogram(np.zeros(1, np.int64), np.zeros(1, np.int64), 4, 4, 3, 4)
    with pytest.raises(capi.InvalidValue):
        mx.block_histogram(np.zeros(1, np.int64), np.zeros(1, np.int64), 4, 4, 512, 4)
    assert mx.block_histogram(np.zeros(0, np.int64), np.zeros(0, np.int64), 4, 4, 2, 2) == {}
