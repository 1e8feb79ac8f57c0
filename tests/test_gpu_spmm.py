"""GPU SpMM: Y += A X for k right-hand sides.  Column j of Y must be bitwise
what abhsf_spmv gives for column j of X (and so, in the reference order,
bitwise the reference CSR's y for that column), whatever the block size, the
schemes, the pass width the ring kernel picks, or the leading dimensions."""
import numpy as np
import pytest

from abhsf_b200 import AbhsfMatrix, capi
from abhsf_b200 import workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu


def _spmm(A, X, Y0, ldx_pad=0, ldy_pad=0):
    """Y0 + A X through abhsf_spmm, X and Y placed in wider row-major buffers
    when a padding is given (ldx = k + ldx_pad)."""
    import torch
    n, k = X.shape
    m = Y0.shape[0]
    Xb = torch.zeros((n, k + ldx_pad), dtype=torch.float64, device="cuda")
    Yb = torch.full((m, k + ldy_pad), 7.0, dtype=torch.float64, device="cuda")
    Xb[:, :k] = torch.from_numpy(X)
    Yb[:, :k] = torch.from_numpy(Y0)
    A.spmm(Xb[:, :k], Yb[:, :k])
    torch.cuda.synchronize()
    out = Yb.cpu().numpy()
    assert np.all(out[:, k:] == 7.0), "abhsf_spmm wrote outside the k columns"
    return out[:, :k]


def _spmv_columns(A, X, Y0):
    import torch
    cols = []
    for j in range(X.shape[1]):
        x = torch.from_numpy(np.ascontiguousarray(X[:, j])).cuda()
        y = torch.from_numpy(np.ascontiguousarray(Y0[:, j])).cuda()
        A.spmv(x, y)
        torch.cuda.synchronize()
        cols.append(y.cpu().numpy())
    return np.stack(cols, axis=1)


def _inputs(coo, k, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, (coo.n, k)), rng.standard_normal((coo.m, k))


@pytest.mark.parametrize("order", ["reference", "tree"])
@pytest.mark.parametrize("s", [16, 32, 64, 128])
@pytest.mark.parametrize("k", [1, 2, 3, 5, 8, 13])
def test_spmm_columns_equal_spmv(gpu, s, k, order):
    coo = W.random_blocky(3000, 2500, s, 200, seed=11)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, sum_order=order)
    X, Y0 = _inputs(coo, k, seed=k)
    Y = _spmm(A, X, Y0)
    np.testing.assert_array_equal(Y, _spmv_columns(A, X, Y0))
    assert A.device_status() == 0


@pytest.mark.parametrize("s", [32, 64])
@pytest.mark.parametrize("forced", ["coo", "csr", "bitmap", "dense"])
def test_spmm_reference_order_all_schemes(gpu, s, forced):
    """Every scheme through the multi-column passes, against the reference
    order per column; forced COO on full tiles only fits narrow passes."""
    coo = W.random_blocky(700, 900, s, 40, seed=5)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, forced_scheme=forced)
    X, Y0 = _inputs(coo, 9, seed=3)
    Y = _spmm(A, X, Y0)
    order = np.lexsort((coo.cols, coo.rows))
    r, c, v = coo.rows[order], coo.cols[order], coo.vals[order]
    for j in range(X.shape[1]):
        np.testing.assert_array_equal(Y[:, j], oracle.spmv_elements(r, c, v, X[:, j].copy(), Y0[:, j].copy()))


def test_spmm_full_dense_tiles_forced_coo(gpu):
    """Fully populated 64 x 64 tiles stored as COO: the largest slot there is;
    the passes fall back to the widths that fit."""
    rows, cols = np.meshgrid(np.arange(128), np.arange(192), indexing="ij")
    rows, cols = rows.ravel().astype(np.int64), cols.ravel().astype(np.int64)
    vals = np.random.default_rng(2).standard_normal(rows.size)
    A = AbhsfMatrix.from_elements(rows, cols, vals, 150, 200, block_size=64, forced_scheme="coo")
    rng = np.random.default_rng(4)
    X, Y0 = rng.uniform(-1, 1, (200, 8)), rng.standard_normal((150, 8))
    np.testing.assert_array_equal(_spmm(A, X, Y0), _spmv_columns(A, X, Y0))


@pytest.mark.parametrize("pads", [(3, 0), (0, 5), (1, 2)])
def test_spmm_leading_dimensions(gpu, pads):
    coo = W.random_blocky(1500, 1700, 64, 120, seed=8)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
    X, Y0 = _inputs(coo, 6, seed=6)
    np.testing.assert_array_equal(_spmm(A, X, Y0, *pads), _spmv_columns(A, X, Y0))


def test_spmm_tiled_mixture_matches_spmv(gpu):
    """The benchmark matrix at a reduced order, k = 16 (two passes of 8 or
    four of 4, whichever fits)."""
    coo = W.tiled_mixture(n=262144)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
    X, Y0 = _inputs(coo, 16, seed=1)
    np.testing.assert_array_equal(_spmm(A, X, Y0), _spmv_columns(A, X, Y0))


@pytest.mark.parametrize("s", [32, 64])
@pytest.mark.parametrize("forced", [None, "coo", "csr", "bitmap", "dense"])
@pytest.mark.parametrize("k", [16, 32, 50])
@pytest.mark.parametrize("pads", [(3, 1), (2, 4), (0, 0)])
def test_spmm_wide_k_every_scheme(gpu, s, forced, k, pads):
    """16, 32 and 50 right-hand sides over every scheme (the ring's passes of
    up to 8 columns, the row slices' passes of up to 32), inside wider rows
    of X and Y: rows whose K values are 16-byte aligned travel as bulk copies
    (pads 2, 4 and 0), the others element by element (pads 3, 1).  Every
    column bitwise its SpMV, and the reference order per column."""
    coo = W.random_blocky(1300, 1500, s, 90, seed=15)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, forced_scheme=forced)
    X, Y0 = _inputs(coo, k, seed=k + s)
    Y = _spmm(A, X, Y0, *pads)
    np.testing.assert_array_equal(Y, _spmv_columns(A, X, Y0))
    order = np.lexsort((coo.cols, coo.rows))
    r, c, v = coo.rows[order], coo.cols[order], coo.vals[order]
    for j in (0, k - 1):
        np.testing.assert_array_equal(Y[:, j], oracle.spmv_elements(r, c, v, X[:, j].copy(), Y0[:, j].copy()))


@pytest.mark.parametrize("s", [16, 32, 64])
@pytest.mark.parametrize("forced", [None, "coo", "csr", "bitmap", "dense"])
@pytest.mark.parametrize("k,pads", [(16, (0, 0)), (32, (2, 6)), (48, (0, 2)), (64, (0, 0))])
def test_spmm_one_pass_every_scheme(gpu, s, forced, k, pads):
    """k a multiple of 16 with X and Y 16-byte aligned and even leading
    dimensions: the wide kernel, 16 or 32 columns a pass with the lanes as
    columns, ragged m and n.  Every column bitwise its SpMV."""
    coo = W.random_blocky(1100, 1300, s, 80, seed=17)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, forced_scheme=forced)
    X, Y0 = _inputs(coo, k, seed=k + s + 1)
    np.testing.assert_array_equal(_spmm(A, X, Y0, *pads), _spmv_columns(A, X, Y0))


@pytest.mark.parametrize("s", [16, 64])
def test_spmm_one_pass_beside_slices(gpu, s):
    """Hypersparse and dense block rows together: the slice SpMM kernels take
    the first, the wide kernel the rest, 32 columns in one pass."""
    coo = W.rmat(1 << 12, 20, seed=5)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s)
    assert A.slices()["slices"] > 0
    X, Y0 = _inputs(coo, 32, seed=s)
    Y = _spmm(A, X, Y0)
    np.testing.assert_array_equal(Y, _spmv_columns(A, X, Y0))
    order = np.lexsort((coo.cols, coo.rows))
    r, c, v = coo.rows[order], coo.cols[order], coo.vals[order]
    np.testing.assert_array_equal(Y[:, 5], oracle.spmv_elements(r, c, v, X[:, 5].copy(), Y0[:, 5].copy()))


def test_spmm_dense_zeros_like_the_spmv(gpu):
    """A dense tile with stored zeros (explicit zero elements among them), 32
    right-hand sides: the SpMM treats them as the SpMV does."""
    rng = np.random.default_rng(3)
    rows, cols = np.meshgrid(np.arange(64), np.arange(64), indexing="ij")
    rows, cols = rows.ravel().astype(np.int64), cols.ravel().astype(np.int64)
    vals = rng.standard_normal(rows.size)
    vals[::7] = 0.0
    A = AbhsfMatrix.from_elements(rows, cols, vals, 100, 90, block_size=64, forced_scheme="dense")
    X, Y0 = rng.uniform(-1, 1, (90, 32)), rng.standard_normal((100, 32))
    np.testing.assert_array_equal(_spmm(A, X, Y0), _spmv_columns(A, X, Y0))


@pytest.mark.parametrize("k", [32, 45])
def test_spmm_power_law_wide_passes(gpu, k):
    """R-MAT (power-law rows): sliced rows and chains through the passes of 32
    (then 8, 4, 1) columns, against the reference order per column."""
    coo = W.rmat(1 << 13, 24, seed=9)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
    sl = A.slices()
    assert sl["slices"] > 0
    X, Y0 = _inputs(coo, k, seed=k)
    Y = _spmm(A, X, Y0, 2, 1)
    order = np.lexsort((coo.cols, coo.rows))
    r, c, v = coo.rows[order], coo.cols[order], coo.vals[order]
    for j in (0, 7, k - 1):
        np.testing.assert_array_equal(Y[:, j], oracle.spmv_elements(r, c, v, X[:, j].copy(), Y0[:, j].copy()))
    np.testing.assert_array_equal(Y, _spmv_columns(A, X, Y0))


def test_spmm_arguments(gpu):
    import torch
    coo = W.random_blocky(300, 200, 64, 10, seed=1)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n)
    X = torch.zeros((200, 4), dtype=torch.float64, device="cuda")
    Y = torch.zeros((300, 4), dtype=torch.float64, device="cuda")
    lib, h = capi.lib, A.handle
    assert lib.abhsf_spmm(h, 4, X.data_ptr(), 3, Y.data_ptr(), 4, None) == capi.INVALID_VALUE
    assert lib.abhsf_spmm(h, 4, X.data_ptr(), 4, Y.data_ptr(), 2, None) == capi.INVALID_VALUE
    assert lib.abhsf_spmm(h, -1, X.data_ptr(), 4, Y.data_ptr(), 4, None) == capi.INVALID_VALUE
    assert lib.abhsf_spmm(h, 4, None, 4, Y.data_ptr(), 4, None) == capi.INVALID_VALUE
    assert lib.abhsf_spmm(h, 0, None, 0, None, 0, None) == capi.SUCCESS
    with pytest.raises(capi.InvalidValue):
        A.spmm(X[:, :3], Y)
