"""Matrix Market ingest with the parse on the GPU (abhsf_read_mtx_device):
the same elements, in the same order, bit for bit, and the same errors as
the host reader abhsf_read_mtx -- itself pinned against the reference's
read_mtx_real_or_binary (include/abhsf/utils/matrix_market_reader.h:146-200;
tests/test_mtx_reader.py) -- on the reference-read fixtures, on generated and
noisy files, and on a large file."""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from abhsf_b200 import capi
from abhsf_b200 import matrix as mx

pytestmark = pytest.mark.gpu

hyp = pytest.importorskip("hypothesis")
st = pytest.importorskip("hypothesis.strategies")

REF = np.load(os.path.join(GOLDEN, "mtx_ref.npz"))
NAMES = sorted({k.split("__")[0] for k in REF.files})


def same(dev, host):
    r, c, v, m, n, info = dev
    hr, hc, hv, hm, hn, hinfo = host
    assert (m, n) == (hm, hn)
    np.testing.assert_array_equal(r.cpu().numpy(), hr)
    np.testing.assert_array_equal(c.cpu().numpy(), hc)
    np.testing.assert_array_equal(v.cpu().numpy().view(np.uint64), hv.view(np.uint64))
    for k in ("matrix_type", "symmetry", "stored_triangle"):
        assert info[k] == hinfo[k], k


def outcome(fn, p):
    try:
        return fn(p), None
    except capi.AbhsfError as e:
        return None, type(e)


def check_file(p):
    h, he = outcome(mx.read_mtx, p)
    d, de = outcome(mx.read_mtx_device, p)
    assert he == de, (he, de)
    if h is not None:
        same(d, h)
    return d


@pytest.mark.parametrize("name", NAMES)
def test_fixtures_equal_the_reference_reader(gpu, name):
    p = os.path.join(GOLDEN, "mtx", name + ".mtx")
    d = mx.read_mtx_device(p)
    assert [d[3], d[4]] == REF[name + "__shape"].tolist()
    np.testing.assert_array_equal(d[0].cpu().numpy(), REF[name + "__rows"])
    np.testing.assert_array_equal(d[1].cpu().numpy(), REF[name + "__cols"])
    np.testing.assert_array_equal(d[2].cpu().numpy().view(np.uint64), REF[name + "__vals"].view(np.uint64))
    check_file(p)


def test_large_file_parsed_on_the_device(gpu, tmp_path):
    rng = np.random.default_rng(5)
    m, n, k = 50000, 60000, 600000
    r = rng.integers(1, m + 1, k)
    c = rng.integers(1, n + 1, k)
    v = rng.standard_normal(k) * 10.0 ** rng.integers(-30, 30, k)
    p = tmp_path / "big.mtx"
    with open(p, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real general\n% a comment\n{m} {n} {k}\n")
        f.write("\n".join(f"{a} {b} {x:.17g}" if i % 3 else f"{a}\t{b}\t{x:.16e}"
                          for i, (a, b, x) in enumerate(zip(r.tolist(), c.tolist(), v.tolist()))))
        f.write("\n")
    d = check_file(str(p))
    assert d[0].numel() == k and d[5]["host_parsed"] == 0


def test_header_longer_than_the_first_chunk(gpu, tmp_path):
    """The file travels to the device in 16 MiB chunks and the banner and
    size line are read from the first; comments past it are read again from
    the whole file."""
    p = tmp_path / "long_header.mtx"
    with open(p, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        for _ in range(18):
            f.write("%" + "c" * (1 << 20) + "\n")
        f.write("3 3 3\n1 1 1.5\n2 2 2.5\n3 3 -3.5\n")
    d = check_file(str(p))
    assert d[0].numel() == 3


def test_other_spellings_go_to_the_host_line_by_line(gpu, tmp_path):
    text = ("%%MatrixMarket matrix coordinate real general\n4 4 6\n"
            "1 1 +2.5\n2 2 0x1p3\n  3 3 1.0000000000000000000001\n\n4 4 1e-320\n1 2 -0\n2 1 7.25 trailing words\n"
            "9 9 these lines are past nnz\n")
    p = tmp_path / "a.mtx"
    p.write_text(text)
    d = check_file(str(p))
    assert d[5]["host_parsed"] == 4 and d[0].numel() == 5  # the zero is dropped


def test_entries_spread_over_lines_read_by_the_host_reader(gpu, tmp_path):
    p = tmp_path / "a.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1\n 2.0\n3 3 4.5\n")
    d = check_file(str(p))
    assert d[0].numel() == 2


@pytest.mark.parametrize("text", [
    "%%MatrixMarket matrix coordinate real symmetric\n3 3 2\n2 1 1\n1 2 1\n",  # both triangles
    "%%MatrixMarket matrix coordinate integer general\n2 2 1\n1 1 3\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n",  # outside m x n
    "%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n2 2 2\n",  # too few
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n1 x 1\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1\n% comment among entries\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 0\n",
    "%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n3 1\n2 2\n",
])
def test_errors_and_edges_as_the_host_reader(gpu, tmp_path, text):
    p = tmp_path / "e.mtx"
    p.write_text(text)
    check_file(str(p))


from test_mtx_reader_fuzz import mtx_files  # noqa: E402  (the generators of the host reader's tests)
from test_reader_robustness import noisy_mtx  # noqa: E402


@hyp.settings(max_examples=120, deadline=None, derandomize=True)
@hyp.given(text=mtx_files())
def test_generated_files(gpu, text):
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "a.mtx")
        with open(p, "w", newline="") as f:
            f.write(text)
        check_file(p)


@hyp.settings(max_examples=200, deadline=None, derandomize=True)
@hyp.given(text=noisy_mtx())
def test_noisy_files(gpu, text):
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "a.mtx")
        with open(p, "w", newline="") as f:
            f.write(text)
        check_file(p)
