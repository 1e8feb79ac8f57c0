"""GPU builder parity: the format arrays the GPU builds are bit-exact against
the CPU oracle builder, and GPU block histograms / mmf totals match the
reference's block_stats + mmf outputs (golden fixtures)."""
import numpy as np
import pytest

from conftest import golden_matrices, golden_stats
from abhsf_b200 import AbhsfMatrix, block_histogram, capi
from abhsf_b200 import workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu

STATS = golden_stats()
MATS = golden_matrices()
ARRAYS = ("brow_ptr", "tile_col", "tile_nnz", "tile_scheme", "tile_val_off", "tile_idx_off")


def assert_same_format(A: AbhsfMatrix, b: "oracle.Built", tag=""):
    e = A.export()
    for k in ARRAYS:
        np.testing.assert_array_equal(e[k], getattr(b, k), err_msg=f"{tag} {k}")
    np.testing.assert_array_equal(e["payload"], b.idx, err_msg=f"{tag} payload")
    np.testing.assert_array_equal(e["values"].view(np.uint8), b.values.view(np.uint8), err_msg=f"{tag} values")


def _mtype(name):
    return STATS[name]["field"] if name in STATS else "real"


@pytest.mark.parametrize("s", [16, 32, 64, 128, 256])
def test_format_bit_exact_minbss(gpu, s):
    for name, coo in MATS.items():
        mt = _mtype(name)
        binary = mt == "pattern"
        vals = None if binary else coo.vals
        for allow in (True, False):
            A = AbhsfMatrix.from_elements(coo.rows, coo.cols, vals, coo.m, coo.n, block_size=s, allow_csr=allow,
                                          matrix_type="binary" if binary else "real")
            b = oracle.build(coo.rows, coo.cols, vals, coo.m, coo.n, s, is_binary=binary, allow_csr=allow)
            assert_same_format(A, b, f"{name} s={s} csr={allow}")
            A.release()


@pytest.mark.parametrize("forced", ["coo", "csr", "bitmap", "dense"])
@pytest.mark.parametrize("s", [16, 64, 256])
def test_format_bit_exact_forced(gpu, s, forced):
    for name in ("rand_real", "blocky64", "blocky16", "edge_ragged_empty_rows", "edge_dense_70", "test_mtx",
                 "edge_one_by_one"):
        coo = MATS[name]
        A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, forced_scheme=forced)
        b = oracle.build(coo.rows, coo.cols, coo.vals, coo.m, coo.n, s,
                         forced_scheme=capi.SCHEME_NAMES.index(forced))
        assert_same_format(A, b, f"{name} s={s} {forced}")
        A.release()


@pytest.mark.parametrize("vt,bits", [("f32", 32), ("bf16", 16)])
def test_format_bit_exact_low_precision_values(gpu, vt, bits):
    for name in ("rand_real", "blocky64", "edge_dense_70"):
        coo = MATS[name]
        A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64, value_type=vt)
        b = oracle.build(coo.rows, coo.cols, coo.vals, coo.m, coo.n, 64, value_type=vt, bits=bits)
        assert_same_format(A, b, f"{name} {vt}")
        A.release()


def test_format_bit_exact_laplace2d_512(gpu):
    c = W.laplacian_2d(512)
    A = AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=64)
    b = oracle.build(c.rows, c.cols, c.vals, c.m, c.n, 64)
    assert_same_format(A, b, "laplace2d_512")
    st = A.stats()
    assert st["tiles"] == 19440
    assert st["tiles_per_scheme"] == {"coo": 7168 + 8176, "csr": 4096, "bitmap": 0, "dense": 0}
    line = [l for l in STATS["laplace2d_512"]["mmf_double"] if l[:2] == [64, 64]][0]
    assert st["msmf_bits"] == line[2:]


def test_stats_msmf_match_reference_mmf(gpu):
    for name, coo in MATS.items():
        g = STATS[name]
        if g["field"] != "real":
            continue
        for s in (16, 32, 64, 128, 256):
            for vt, key in (("f64", "mmf_double"), ("f32", "mmf_single")):
                A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, value_type=vt)
                line = [l for l in g[key] if l[:2] == [s, s]][0]
                assert A.stats()["msmf_bits"] == line[2:], (name, s, vt)
                A.release()


def test_gpu_block_histograms_match_reference(gpu):
    import torch
    for name, g in STATS.items():
        coo = W.laplacian_2d(512) if name == "laplace2d_512" else MATS[name]
        dev_rows = torch.from_numpy(coo.rows).cuda()
        dev_cols = torch.from_numpy(coo.cols).cuda()
        for rs, hist in g["bstats"].items():
            r, s = (int(t) for t in rs.split("x"))
            want = {int(z): c for z, c in hist.items()}
            assert block_histogram(coo.rows, coo.cols, coo.m, coo.n, r, s) == want, (name, rs)
            if r == s:
                assert block_histogram(dev_rows, dev_cols, coo.m, coo.n, r, s) == want, (name, rs)


def test_builder_errors(gpu):
    with pytest.raises(capi.DuplicateEntry):
        AbhsfMatrix.from_elements(np.array([0, 3, 0]), np.array([1, 2, 1]), np.ones(3), 4, 4, block_size=16)
    with pytest.raises(capi.IndexOutOfRange):
        AbhsfMatrix.from_elements(np.array([0, 4]), np.array([1, 1]), np.ones(2), 4, 4, block_size=16)
    with pytest.raises(capi.IndexOutOfRange):
        AbhsfMatrix.from_elements(np.array([0, -1]), np.array([1, 1]), np.ones(2), 4, 4, block_size=16)
    # a full 256 x 256 tile cannot be CSR (uint16 row_end)
    r, c = np.divmod(np.arange(256 * 256, dtype=np.int64), 256)
    with pytest.raises(capi.Unsupported):
        AbhsfMatrix.from_elements(r, c, np.ones(r.size), 256, 256, block_size=256, forced_scheme="csr")
    # the handle remains usable after errors: a valid build succeeds
    A = AbhsfMatrix.from_elements(np.array([0]), np.array([0]), np.ones(1), 1, 1, block_size=16)
    assert A.stats()["tiles"] == 1


def test_empty_matrix(gpu):
    import torch
    A = AbhsfMatrix.from_elements(np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0), 100, 70, block_size=32)
    st = A.stats()
    assert st["tiles"] == 0 and st["block_rows"] == 4
    x = torch.ones(70, dtype=torch.float64, device="cuda")
    y = torch.full((100,), 2.0, dtype=torch.float64, device="cuda")
    A.spmv(x, y)
    torch.cuda.synchronize()
    assert torch.all(y == 2.0)


@pytest.mark.parametrize("name", sorted(golden_stats()))
def test_all_block_sizes_in_one_call_match_reference_block_stats(gpu, name):
    """abhsf_block_histogram_all: the 64 .bstats histograms of the reference's
    block_stats (block_statistics/block_stats.cpp:144-170) from one call."""
    from abhsf_b200 import block_histograms_all
    g = golden_stats()[name]
    coo = W.laplacian_2d(512) if name == "laplace2d_512" else golden_matrices()[name]
    got = block_histograms_all(coo.rows, coo.cols, coo.m, coo.n)
    want = {rs: {int(z): c for z, c in h.items()} for rs, h in g["bstats"].items()}
    assert set(got) == set(want)
    for rs in want:
        assert got[rs] == want[rs], rs


def test_all_block_sizes_equal_per_size_histograms(gpu):
    import torch
    from abhsf_b200 import block_histogram, block_histograms_all
    coo = W.tiled_mixture(n=65536 + 37, p=1e-3, seed=5)
    for rows, cols in ((coo.rows, coo.cols), (torch.from_numpy(coo.rows).cuda(), torch.from_numpy(coo.cols).cuda())):
        got = block_histograms_all(rows, cols, coo.m, coo.n)
        for rs, h in got.items():  # conservation, block_statistics/block_stats.cpp:165-168
            assert sum(z * c for z, c in h.items()) == coo.nnz, rs
        for rs in ("2x2", "4x256", "64x64", "256x2", "256x256", "128x32"):
            r, s = (int(t) for t in rs.split("x"))
            assert got[rs] == block_histogram(coo.rows, coo.cols, coo.m, coo.n, r, s), rs
    with pytest.raises(capi.IndexOutOfRange):
        block_histograms_all(np.array([0, 9]), np.array([0, 1]), 5, 5)
    empty = block_histograms_all(np.zeros(0, np.int64), np.zeros(0, np.int64), 5, 5)
    assert all(h == {} for h in empty.values())
