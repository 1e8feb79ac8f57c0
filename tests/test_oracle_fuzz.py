"""The oracle's block histograms and the library's mmf lines against the
reference's own block_stats and mmf programs (compiled from the reference
sources into oracle/_ref/, the checker) on generated matrices: random sizes
up to 600 x 600, elements scattered, clustered into a few tiles (dense and
bitmap tiles) or laid along bands, for all 64 block sizes.  Without the
reference programs the test is skipped; the committed golden fixtures cover
the same comparison on fixed matrices."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from abhsf_b200 import matrix as mx
from oracle import oracle

hyp = pytest.importorskip("hypothesis")
st = pytest.importorskip("hypothesis.strategies")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
pytestmark = pytest.mark.skipif(
    not all(os.path.exists(os.path.join(REF_DIR, p)) for p in ("block_stats", "mmf")),
    reason="reference block_stats / mmf not built (make -C oracle ref)")


@st.composite
def matrices(draw):
    m = draw(st.integers(1, 600))
    n = draw(st.integers(1, 600))
    kind = draw(st.sampled_from(["scatter", "cluster", "band"]))
    seed = draw(st.integers(0, 2 ** 31 - 1))
    rng = np.random.default_rng(seed)
    k = draw(st.integers(1, 3000))
    if kind == "scatter":
        key = rng.integers(0, m * n, k)
    elif kind == "cluster":  # a few dense corners: 1..64 x 1..64 windows filled at random density
        keys = []
        for _ in range(draw(st.integers(1, 4))):
            h, w = rng.integers(1, 65, 2)
            r0, c0 = rng.integers(0, m), rng.integers(0, n)
            rr, cc = np.meshgrid(np.arange(r0, min(r0 + h, m)), np.arange(c0, min(c0 + w, n)), indexing="ij")
            win = (rr * n + cc).reshape(-1)
            keys.append(win[rng.random(win.size) < rng.uniform(0.2, 1.0)])
        key = np.concatenate(keys + [rng.integers(0, m * n, 5)])
    else:
        i = rng.integers(0, m, k)
        j = np.clip(i * n // m + rng.integers(-8, 9, k), 0, n - 1)
        key = i * n + j
    key = np.unique(key)
    vals = rng.standard_normal(key.size)
    vals[vals == 0] = 1.0
    return m, n, key // n, key % n, vals


def reference_stats(m, n, rows, cols, vals, d):
    p = os.path.join(d, "a.mtx")
    with open(p, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real general\n{m} {n} {rows.size}\n")
        f.write("".join(f"{i + 1} {j + 1} {v:.17g}\n" for i, j, v in zip(rows, cols, vals)))
    subprocess.run([os.path.join(REF_DIR, "block_stats"), p], cwd=d, check=True, stdout=subprocess.DEVNULL)
    subprocess.run([os.path.join(REF_DIR, "mmf")], cwd=d, check=True, stdout=subprocess.DEVNULL)
    props = [int(t) for t in open(os.path.join(d, "props")).read().split()]
    hists = {}
    for k in range(1, 9):
        for l in range(1, 9):
            h = {}
            for line in open(os.path.join(d, f"{1 << k}x{1 << l}.bstats")):
                z, c = line.split()
                h[int(z)] = int(c)
            hists[(k, l)] = h
    mmf = {prec: {(t[0], t[1]): t[2:] for t in ([int(v) for v in line.split()]
                                                 for line in open(os.path.join(d, "mmf-" + prec)) if line.strip())}
           for prec in ("single", "double")}
    return props, hists, mmf


@hyp.settings(max_examples=60, deadline=None, derandomize=True)
@hyp.given(mat=matrices())
def test_generated_matrices_match_block_stats_and_mmf(mat):
    m, n, rows, cols, vals = mat
    with tempfile.TemporaryDirectory() as d:
        props, hists, mmf = reference_stats(m, n, rows, cols, vals, d)
    assert props[:4] == [m, n, rows.size, rows.size]
    for (k, l), h in hists.items():
        assert oracle.block_histogram(rows, cols, k, l) == h, (k, l)
        assert sum(z * c for z, c in h.items()) == rows.size
        r, s = 1 << k, 1 << l
        o1, o2 = mx.mmf_line(m, n, rows.size, "real", r, s, h)
        assert o1 == mmf["single"][(r, s)] and o2 == mmf["double"][(r, s)], (r, s)
        assert (o1, o2) == tuple(oracle.mmf_line(m, n, rows.size, 2, r, s, h))


@pytest.mark.skipif(not oracle.RefCSR.available(), reason="reference CSR not built (make -C oracle ref)")
@hyp.settings(max_examples=60, deadline=None, derandomize=True)
@hyp.given(mat=matrices(), s=st.sampled_from([16, 32, 64, 128, 256]), seed=st.integers(0, 1000))
def test_generated_matrices_spmv_bits_match_reference_csr(mat, s, seed):
    """y from the reference's CSR spmv_naive (spmv/bottlenecks/spmv.cpp:58-64),
    from the oracle's element loop on row-major elements, and from the oracle's
    ABHSF format at block size s (serial and on all host threads): the same
    bits, with random values, x and y."""
    m, n, rows, cols, vals = mat
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, n)
    y0 = rng.standard_normal(m)
    ref = oracle.RefCSR(rows, cols, vals, m, n)
    y_ref = y0.copy()
    ref.spmv(x, y_ref)
    ref.release()
    y_loop = oracle.spmv_elements(rows, cols, vals, x, y0.copy())  # rows, cols come row-major from np.unique
    np.testing.assert_array_equal(y_loop, y_ref)
    b = oracle.build(rows, cols, vals, m, n, s)
    y_fmt = y0.copy()
    b.spmv(x, y_fmt)
    np.testing.assert_array_equal(y_fmt, y_ref)
    y_omp = y0.copy()
    b.spmv_omp(x, y_omp)
    np.testing.assert_array_equal(y_omp, y_ref)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "min-bss")), reason="reference min-bss not built")
@hyp.settings(max_examples=8, deadline=None, derandomize=True)
@hyp.given(mats=st.lists(matrices(), min_size=1, max_size=4))
def test_generated_matrices_match_min_bss(mats):
    """The reference's min-bss over several matrices at once (one directory
    each, as block_statistics/min-bss.cpp reads them): its mmf-bss-single /
    -double columns equal selector.min_bss of the library's mmf table, and
    block_opt is the least of them."""
    from abhsf_b200 import selector
    with tempfile.TemporaryDirectory() as d:
        ours = {}
        for i, (m, n, rows, cols, vals) in enumerate(mats):
            sub = os.path.join(d, f"m{i}")
            os.mkdir(sub)
            reference_stats(m, n, rows, cols, vals, sub)
            hists = {f"{1 << k}x{1 << l}": oracle.block_histogram(rows, cols, k, l)
                     for k in range(1, 9) for l in range(1, 9)}
            ours[f"m{i}"] = selector.mmf_table(hists, m, n, rows.size)
        subprocess.run([os.path.join(REF_DIR, "min-bss")], cwd=d, check=True, stdout=subprocess.DEVNULL)
        for prec in ("single", "double"):
            text = open(os.path.join(d, "mmf-bss-" + prec)).read().split("\n")
            names = text[0].split()[2:]
            assert names == sorted(ours)
            ref = {}
            for line in text[1:]:
                t = line.split()
                if t:
                    ref[(int(t[0]), int(t[1]))] = [int(v) for v in t[2:]]
            assert len(ref) == 64
            for j, name in enumerate(names):
                mb = selector.min_bss(ours[name], prec)
                assert list(mb) == sorted(ref)
                assert [mb[bs] for bs in sorted(ref)] == [ref[bs][j] for bs in sorted(ref)]
                (h, w), col, bits = selector.block_opt(ours[name], prec)
                assert bits == min(mb.values()) and mb[(h, w)] == bits
                first = next(bs for bs in sorted(mb) if mb[bs] == bits)  # strict '<': the first size wins
                assert (h, w) == first
                assert ours[name][(h, w)][{"single": 0, "double": 1}[prec]][selector.MMF_COLUMNS.index(col)] == bits


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "consistency")), reason="reference consistency not built")
@hyp.settings(max_examples=6, deadline=None, derandomize=True)
@hyp.given(mats=st.lists(matrices(), min_size=2, max_size=5))
def test_generated_matrices_match_consistency(mats):
    """The reference's consistency program over all the matrices (both
    schemes, both precisions): its B_64 / B_20 / B_14 / B_8 average and
    maximum excess equal selector.consistency of the library's mmf tables
    (to the 6 digits it prints)."""
    import re

    from abhsf_b200 import selector
    with tempfile.TemporaryDirectory() as d:
        tables = []
        for i, (m, n, rows, cols, vals) in enumerate(mats):
            sub = os.path.join(d, f"m{i}")
            os.mkdir(sub)
            reference_stats(m, n, rows, cols, vals, sub)
            hists = {f"{1 << k}x{1 << l}": oracle.block_histogram(rows, cols, k, l)
                     for k in range(1, 9) for l in range(1, 9)}
            tables.append(selector.mmf_table(hists, m, n, rows.size))
        for scheme, sname in ((0, "min-fixed"), (1, "adaptive")):
            for prec, pname in ((0, "single"), (1, "double")):
                r = subprocess.run([os.path.join(REF_DIR, "consistency"), str(scheme), str(prec), str(len(mats))],
                                   cwd=d, check=True, capture_output=True, text=True)
                text = re.sub(r"\x1b\[[0-9;]*m", "", r.stdout)
                ref = {k: (float(a), float(b)) for k, a, b in
                       re.findall(r"(B_\d+): Average = ([0-9.eE+-]+), Maximum = ([0-9.eE+-]+)", text)}
                ours = selector.consistency(tables, sname, pname)
                assert set(ref) == set(ours)
                for k in ref:
                    for a, b in zip(ours[k], ref[k]):
                        assert abs(a - b) <= 1e-5 * max(abs(b), 1e-3), (sname, pname, k, ours[k], ref[k])


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "min-schemes")), reason="reference min-schemes not built")
@hyp.settings(max_examples=6, deadline=None, derandomize=True)
@hyp.given(mats=st.lists(matrices(), min_size=1, max_size=4))
def test_generated_matrices_match_min_schemes(mats):
    """The reference's min-schemes lines (each column's least storage over
    the 64 sizes, and block_opt's size) equal selector.min_schemes."""
    from abhsf_b200 import selector
    with tempfile.TemporaryDirectory() as d:
        ours = {}
        for i, (m, n, rows, cols, vals) in enumerate(mats):
            sub = os.path.join(d, f"m{i}")
            os.mkdir(sub)
            reference_stats(m, n, rows, cols, vals, sub)
            hists = {f"{1 << k}x{1 << l}": oracle.block_histogram(rows, cols, k, l)
                     for k in range(1, 9) for l in range(1, 9)}
            ours[f"m{i}"] = selector.mmf_table(hists, m, n, rows.size)
        subprocess.run([os.path.join(REF_DIR, "min-schemes")], cwd=d, check=True, stdout=subprocess.DEVNULL)
        for prec in ("single", "double"):
            lines = [l.split() for l in open(os.path.join(d, "mmf-schemes-" + prec)) if l.strip()]
            assert sorted(l[0] for l in lines) == sorted(ours)
            for l in lines:
                mins, (h, w) = selector.min_schemes(ours[l[0]], prec)
                assert [int(v) for v in l[1:9]] == mins
                assert (int(l[9]), int(l[10])) == (h, w)


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_DIR, "rows-nnz-stdev")), reason="rows-nnz-stdev not built")
@hyp.settings(max_examples=20, deadline=None, derandomize=True)
@hyp.given(mat=matrices())
def test_generated_matrices_row_stdev_matches_rows_nnz_stdev(mat):
    """The selector's row-count feature is the population standard deviation
    the reference's rows-nnz-stdev prints (from block_stats' rows_nnz_stored),
    to the 6 digits it prints; also as a share of n."""
    from oracle import selector_oracle
    m, n, rows, cols, vals = mat
    with tempfile.TemporaryDirectory() as d:
        reference_stats(m, n, rows, cols, vals, d)
        r = subprocess.run([os.path.join(REF_DIR, "rows-nnz-stdev")], cwd=d, check=True, capture_output=True,
                           text=True)
    ref_stored, ref_all, ref_pct, _ = (float(t) for t in r.stdout.split())
    std = 2.0 ** selector_oracle.features(rows, cols, m, n)[3] - 1.0
    assert abs(std - ref_stored) <= 1e-5 * ref_stored + 1e-9
    assert ref_all == ref_stored  # general matrices: nothing mirrored
    assert abs(std / n * 100.0 - ref_pct) <= 1e-5 * ref_pct + 1e-9
