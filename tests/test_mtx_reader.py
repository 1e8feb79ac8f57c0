"""Matrix Market ingest (abhsf_read_mtx, host code of the library) against
what the reference's own reader, read_mtx_real_or_binary, read from the same
files (tests/golden/mtx_ref.npz, written by tests/golden/make_mtx_golden.py
with the reference reader compiled from its sources)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from abhsf_b200 import capi
from abhsf_b200 import matrix as mx

REF = np.load(os.path.join(GOLDEN, "mtx_ref.npz"))
NAMES = sorted({k.split("__")[0] for k in REF.files})


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("threads", [1, 4])
def test_reader_matches_reference_reader(name, threads):
    rows, cols, vals, m, n, info = mx.read_mtx(os.path.join(GOLDEN, "mtx", name + ".mtx"), threads)
    assert [m, n] == REF[name + "__shape"].tolist()
    np.testing.assert_array_equal(rows, REF[name + "__rows"])
    np.testing.assert_array_equal(cols, REF[name + "__cols"])
    np.testing.assert_array_equal(vals.view(np.uint64), REF[name + "__vals"].view(np.uint64))  # bit for bit
    if "symmetric" in name:
        assert info["symmetry"] == "symmetric" and info["stored_triangle"] in ("lower", "upper")
    if "pattern" in name:
        assert info["matrix_type"] == "binary" and np.all(vals == 1.0)


def test_many_threads_read_a_large_file_in_order(tmp_path):
    rng = np.random.default_rng(3)
    m, n, k = 20000, 30000, 400000
    r = rng.integers(1, m + 1, k)
    c = rng.integers(1, n + 1, k)
    v = rng.standard_normal(k)
    p = tmp_path / "big.mtx"
    with open(p, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real general\n{m} {n} {k}\n")
        f.write("\n".join(f"{a} {b} {x:.17g}" for a, b, x in zip(r, c, v)) + "\n")
    one = mx.read_mtx(str(p), 1)
    many = mx.read_mtx(str(p), 8)
    for a, b in zip(one[:3], many[:3]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(one[0], r - 1)
    np.testing.assert_array_equal(one[1], c - 1)
    np.testing.assert_array_equal(one[2], v)


@pytest.mark.parametrize("text,exc", [
    ("%%MatrixMarket matrix coordinate real symmetric\n3 3 2\n2 1 1\n1 2 1\n", capi.InvalidValue),  # both triangles
    ("%%MatrixMarket matrix coordinate integer general\n2 2 1\n1 1 3\n", capi.Unsupported),
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", capi.Unsupported),
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n", capi.IndexOutOfRange),
    ("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n2 2 2\n", capi.InvalidValue),  # too few
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 x 1\n", capi.InvalidValue),
    ("not a banner\n", capi.InvalidValue),
])
def test_reader_errors(tmp_path, text, exc):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(exc):
        mx.read_mtx(str(p))


def test_missing_file():
    with pytest.raises(capi.InvalidValue):
        mx.read_mtx("/nonexistent/file.mtx")


@pytest.mark.parametrize("threads", [1, 4])
def test_size_line_without_line_end(tmp_path, threads):
    """A file that ends on its size line: no elements (nnz 0), or too few."""
    p = tmp_path / "a.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n1 1 0")
    rows, cols, vals, m, n, _ = mx.read_mtx(str(p), threads)
    assert rows.size == cols.size == vals.size == 0 and (m, n) == (1, 1)
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 3 2")
    with pytest.raises(capi.InvalidValue):
        mx.read_mtx(str(p), threads)
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 3 1\n2 3 4.5")  # last entry without line end
    rows, cols, vals, _, _, _ = mx.read_mtx(str(p), threads)
    assert rows.tolist() == [1] and cols.tolist() == [2] and vals.tolist() == [4.5]


def test_expand_symmetric_counts_like_block_stats():
    """The mirrored element count equals block_stats' "nnz_all" (props
    field 5) for the golden symmetric matrix; skew negates the mirror; the
    stored triangle of the fixture file expands to the full matrix."""
    import json

    from conftest import golden_matrices
    props = json.load(open(os.path.join(GOLDEN, "block_stats.json")))["sym_lower"]["props"]
    coo = golden_matrices()["sym_lower"]
    r, c, v = mx.expand_symmetric(coo.rows, coo.cols, coo.vals, "symmetric")
    assert (coo.nnz, r.size) == (props[3], props[4]) == (1293, 2576)
    dense = np.zeros((coo.m, coo.n))
    dense[r, c] = v
    np.testing.assert_array_equal(dense, dense.T)
    assert np.all(np.diff(r * coo.n + c) > 0)  # row-major, no duplicates
    r, c, v = mx.expand_symmetric(coo.rows, coo.cols, coo.vals, "skew")
    dense = np.zeros((coo.m, coo.n))
    dense[r, c] = v
    off = ~np.eye(coo.m, dtype=bool)
    np.testing.assert_array_equal(dense[off], -dense.T[off])
    rows, cols, vals, m, n, info = mx.read_mtx(os.path.join(GOLDEN, "mtx", "real_symmetric_lower.mtx"))
    r, c, v = mx.expand_symmetric(rows, cols, vals, info["symmetry"])
    assert r.size == 2 * rows.size - int((rows == cols).sum())
    g = mx.expand_symmetric(rows, cols, vals, "general")
    assert g[0] is not None and g[0].size == rows.size
    with pytest.raises(ValueError):
        mx.expand_symmetric(rows, cols, vals, "upper")
