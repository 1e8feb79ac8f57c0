"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from the reference's block_stats, mmf and CSR
spmv_naive, compiled from the reference sources)."""
import numpy as np
import pytest

from conftest import golden_matrices, golden_spmv, golden_stats
from oracle import oracle
from abhsf_b200 import workloads as W

STATS = golden_stats()
MATS = golden_matrices()


def _coo(name):
    if name == "laplace2d_512":
        return W.laplacian_2d(512)
    return MATS[name]


@pytest.mark.parametrize("name", sorted(STATS))
def test_histograms_match_reference_block_stats(name):
    coo = _coo(name)
    g = STATS[name]
    assert g["props"][3] == coo.nnz
    for rs, hist in g["bstats"].items():
        r, s = (int(t) for t in rs.split("x"))
        h = oracle.block_histogram(coo.rows, coo.cols, r.bit_length() - 1, s.bit_length() - 1)
        assert h == {int(z): c for z, c in hist.items()}, rs


@pytest.mark.parametrize("name", sorted(STATS))
def test_mmf_lines_match_reference_mmf(name):
    g = STATS[name]
    m, n, _, nnz_stored, _, mtype, _ = g["props"]
    for line1, line2 in zip(g["mmf_single"], g["mmf_double"]):
        r, s = line1[0], line1[1]
        hist = {int(z): c for z, c in g["bstats"][f"{r}x{s}"].items()}
        o1, o2 = oracle.mmf_line(m, n, nnz_stored, mtype, r, s, hist)
        assert o1 == line1[2:] and o2 == line2[2:], (r, s)


def test_known_answers_laplace2d_512():
    g = STATS["laplace2d_512"]
    assert g["props"] == [262144, 262144, 1308672, 1308672, 1308672, 2, 3]
    assert g["bstats"]["64x64"] == {"1": 7168, "64": 8176, "190": 4096}
    line = [l for l in g["mmf_double"] if l[:2] == [64, 64]][0]
    assert line[2:] == [167510016, 134021152, 99978880, 106823488, 163667776, 5096365888, 98444896, 100017760]
    assert STATS["test_mtx"]["props"] == [6, 7, 15, 15, 15, 2, 3]


def test_oracle_spmv_matches_reference_csr_bitwise():
    """Element-order FP64 loop on row-major sorted elements reproduces the
    reference CSR spmv_naive bit for bit (same additions in the same order)."""
    ref = golden_spmv()
    checked = 0
    for name, coo in MATS.items():
        if name + "__y" not in ref:
            continue
        order = np.lexsort((coo.cols, coo.rows))
        y = ref[name + "__y0"].copy()
        oracle.spmv_elements(coo.rows[order], coo.cols[order], coo.vals[order], ref[name + "__x"], y)
        np.testing.assert_array_equal(y, ref[name + "__y"], err_msg=name)
        checked += 1
    assert checked >= 6
    c1 = W.laplacian_2d(512)
    y = np.zeros(c1.m)
    oracle.spmv_elements(c1.rows, c1.cols, c1.vals, W.rhs(c1.n, 0), y)
    np.testing.assert_array_equal(y, ref["laplace2d_512__y_seed0"])


def test_scheme_crossovers_s64_f64():
    """s = 64, 64-bit values: COO up to 126, CSR 127..554, bitmap 555..4032,
    dense from 4033 (msmf.h, ties to the earlier scheme)."""
    sel = [oracle.select_scheme(64, 64, z, 64) for z in range(1, 4097)]
    assert sel[:126] == [oracle.COO] * 126
    assert sel[126:554] == [oracle.CSR] * (554 - 126)
    assert sel[554:4032] == [oracle.BITMAP] * (4032 - 554)
    assert sel[4032:] == [oracle.DENSE] * (4096 - 4032)
    assert oracle.select_scheme(64, 64, 4096, 64, is_binary=True) == oracle.BITMAP
    assert oracle.select_scheme(64, 64, 300, 64, allow_csr=False) == oracle.COO
    assert oracle.select_scheme(64, 64, 400, 64, allow_csr=False) == oracle.BITMAP


def test_scheme_ties_keep_earlier():
    # find exact ties and check the order COO > CSR > bitmap > dense
    ties = 0
    for s in (2, 4, 8, 16, 32, 64, 128, 256):
        for r in (2, 8, 64, 256):
            for z in range(1, r * s + 1, max(1, r * s // 997)):
                c = {k: oracle.block_bits(k, r, s, z, 64) for k in range(4)}
                best = min(c.values())
                first = [k for k in range(4) if c[k] == best][0]
                assert oracle.select_scheme(r, s, z, 64) == first
                ties += sum(1 for v in c.values() if v == best) > 1
    # the tie rule is exercised at least once over this sweep
    assert ties >= 1


@pytest.mark.parametrize("s", [16, 32, 64, 128, 256])
def test_oracle_builder_roundtrip(s):
    """The CPU builder's arrays decode back to the same y (any scheme)."""
    for name in ("rand_real", "blocky64", "blocky16", "edge_ragged_empty_rows", "edge_dense_70", "test_mtx"):
        coo = MATS[name]
        x = W.rhs(coo.n, 1)
        ref = oracle.spmv_elements(coo.rows, coo.cols, coo.vals, x, np.zeros(coo.m))
        scale = oracle.abs_spmv(coo.rows, coo.cols, coo.vals, x, coo.m)
        for forced in (-1, 0, 1, 2, 3):
            b = oracle.build(coo.rows, coo.cols, coo.vals, coo.m, coo.n, s, forced_scheme=forced)
            y = np.zeros(coo.m)
            b.spmv(x, y)
            assert np.all(np.abs(y - ref) <= 1e-13 * scale), (name, s, forced)
            assert int(b.tile_nnz.sum()) == coo.nnz
            assert b.brow_ptr[-1] == b.T and np.all(np.diff(b.brow_ptr) >= 0)
            assert np.all(b.tile_idx_off % 16 == 0)


def test_oracle_builder_errors():
    with pytest.raises(ValueError, match="duplicate"):
        oracle.build([0, 0], [1, 1], [1.0, 2.0], 4, 4, 16)
    with pytest.raises(ValueError, match="range"):
        oracle.build([0, 4], [1, 1], [1.0, 2.0], 4, 4, 16)


def test_bf16_conversion_rne():
    assert oracle.lib().orc_f64_to_bf16.restype is not None or True
    vals = np.array([1.0, -2.5, 1.00390625, 1.01171875, 3.14159265358979, 1e-40, 65504.0])
    for v in vals:
        b = oracle.build([0], [0], [v], 1, 1, 16, value_type="bf16").values[0]
        f32 = np.float32(v)
        u = int(f32.view(np.uint32))
        want = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF
        assert int(b) == want, v


@pytest.mark.parametrize("s", [16, 64, 256])
def test_oracle_openmp_abhsf_spmv_equals_serial(s):
    """The OpenMP ABHSF SpMV (a CPU baseline) gives the serial oracle's y bit
    for bit: block rows write disjoint rows."""
    for name in ("blocky64", "rand_real", "edge_ragged_empty_rows"):
        coo = MATS[name]
        b = oracle.build(coo.rows, coo.cols, coo.vals, coo.m, coo.n, s)
        x = W.rhs(coo.n, 3)
        y1 = W.rhs(coo.m, 4)
        y2 = y1.copy()
        b.spmv(x, y1)
        b.spmv_omp(x, y2)
        np.testing.assert_array_equal(y1, y2)
    assert oracle.Built.threads() >= 1
