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
    assert C.sizeof(capi.Stats) == 216


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


def test_selection_entry_points_reject_bad_arguments_before_device_work():
    """The block-size selection and MLP entry points check their arguments
    on the host (no GPU needed to see the error)."""
    one = np.zeros(1, np.int64)
    ms = np.zeros(5, np.float32)
    best = C.c_int32()
    fp = C.POINTER(C.c_float)
    # autotune: candidate mask outside the five sizes, non-positive reps, bad shape
    for cand, reps, m in ((32, 1, 4), (-1, 1, 4), (1, 0, 4), (1, 1, 0)):
        st = capi.lib.abhsf_autotune(one.ctypes.data, one.ctypes.data, None, 1, m, 4, None, cand, reps, None,
                                     ms.ctypes.data_as(fp), C.byref(best), None)
        assert st == capi.INVALID_VALUE, (cand, reps, m)
    assert capi.lib.abhsf_autotune(one.ctypes.data, one.ctypes.data, None, 1, 4, 4, None, 0, 1, None, None,
                                   C.byref(best), None) == capi.INVALID_VALUE
    # the storage sweep and the all-sizes histograms need their output arrays
    assert capi.lib.abhsf_block_size_storage(one.ctypes.data, one.ctypes.data, 1, 4, 4, None, None, None,
                                             None) == capi.INVALID_VALUE
    assert capi.lib.abhsf_block_histogram_all(one.ctypes.data, one.ctypes.data, 1, 4, 4, 0, None, None,
                                              None) == capi.INVALID_VALUE
    assert capi.lib.abhsf_block_size_storage(one.ctypes.data, one.ctypes.data, 1, 0, 4, None, None,
                                             np.zeros(5, np.uint64).ctypes.data_as(capi._u64p),
                                             None) == capi.INVALID_VALUE
    # the selector and the MLP kernels
    assert capi.lib.abhsf_selector_predict(None, None, None, C.byref(best)) == capi.INVALID_VALUE
    assert capi.lib.abhsf_selector_predict(None, ms.ctypes.data_as(fp), None, None) == capi.INVALID_VALUE
    assert capi.lib.abhsf_selector_builtin_model(None) == capi.INVALID_VALUE
    assert capi.lib.abhsf_selector_features(one.ctypes.data, one.ctypes.data, 1, 0, 4, 0, None,
                                            ms.ctypes.data_as(fp)) == capi.INVALID_VALUE
    assert capi.lib.abhsf_mlp_forward(None, None, -1, None, None, None) == capi.INVALID_VALUE
    assert capi.lib.abhsf_mlp_backward(None, None, None, 0, None, None, None, None, None, None) == capi.INVALID_VALUE
    assert capi.lib.abhsf_mlp_adam(None, None, None, None, 1, 1e-3, None) == capi.INVALID_VALUE
    assert capi.lib.abhsf_last_error_string()


def test_selector_option_defaults_and_struct():
    o = capi.BuildOpts()
    capi.lib.abhsf_build_opts_default(C.byref(o))
    assert o.block_size == 64 and o.selector == capi.SELECTORS["minbss"] and o.selector_model is None
    assert o.slice_tile_nnz == 0


def test_cost_model_exhaustive_small_blocks():
    """Every (r, s) with r, s <= 16 and every block nonzero count 1 .. r*s:
    the library's scheme costs and choices equal the oracle's restatement of
    include/abhsf/msmf.h:9-63, for f64 and f32 widths, with and without CSR."""
    for r in (2, 4, 8, 16):
        for s in (2, 4, 8, 16):
            for z in range(1, r * s + 1):
                for bits in (64, 32):
                    for sch in range(4):
                        assert mx.block_scheme_bits(sch, r, s, z, bits) == oracle.block_bits(sch, r, s, z, bits)
                    for binary in (False, True):
                        for allow in (False, True):
                            got = mx.block_select_scheme(r, s, z, bits, binary, allow)
                            assert capi.SCHEME_NAMES.index(got) == oracle.select_scheme(r, s, z, bits, binary,
                                                                                        allow), (r, s, z)

