"""Delta-coded row slices: the reference-order SpMV's path for hypersparse
block rows (abhsf_build_opts.slice_tile_nnz).  The slices the GPU builds
equal the oracle's restatement word for word, and y is bitwise the reference
CSR's order for every threshold, with one-row chains (rows of more than 256
elements), bitmap tiles inside slice block rows, f32 / bf16 values, several
right-hand sides, batches and the host-memory pipeline."""
import numpy as np
import pytest

from abhsf_b200 import AbhsfBatch, AbhsfMatrix
from abhsf_b200 import workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu

DEFAULT_TILE_NNZ = 32


def heavy_rows(n=200000, heavy=(0, 1, 5, 70), per_heavy=5000, sparse=200000, seed=0) -> W.Coo:
    """A few rows of per_heavy elements (each summed as a chain) over a
    hypersparse rest."""
    rng = np.random.default_rng(seed)
    r = [np.full(per_heavy, h, np.int64) for h in heavy]
    c = [rng.choice(n, per_heavy, replace=False) for _ in heavy]
    r.append(rng.integers(0, n, sparse))
    c.append(rng.integers(0, n, sparse))
    rows, cols = np.concatenate(r), np.concatenate(c)
    key = np.unique(rows * n + cols)
    rows, cols = key // n, key % n
    return W.Coo(rows, cols, rng.standard_normal(rows.size), n, n, "heavy_rows")


def bitmap_in_sparse_rows(seed=0) -> W.Coo:
    """Block rows whose one dense tile (a bitmap) sits among many single
    elements: a slice block row holding a bitmap tile."""
    rng = np.random.default_rng(seed)
    n = 64 * 300
    rows, cols = [], []
    for I in range(0, 300, 3):
        dense = rng.random((64, 64)) < 0.3
        r, c = np.nonzero(dense)
        rows.append(I * 64 + r)
        cols.append(((I * 7) % 300) * 64 + c)
        rows.append(I * 64 + rng.integers(0, 64, 150))
        cols.append(rng.integers(0, n, 150))
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    key = np.unique(rows * n + cols)
    rows, cols = key // n, key % n
    return W.Coo(rows, cols, rng.standard_normal(rows.size), n, n, "bitmap_in_sparse_rows")


def cases():
    return [W.rmat(1 << 14, 8, seed=3), heavy_rows(), bitmap_in_sparse_rows(), W.tiled_mixture(n=1 << 18),
            W.banded(5000, 3, seed=1), W.random_uniform(3000, 4000, 9000, seed=5)]


def reference_y(coo, x, y0):
    order = np.lexsort((coo.cols, coo.rows))
    return oracle.spmv_elements(coo.rows[order], coo.cols[order], coo.vals[order], x, y0.copy())


def _spmv(A, x, y0):
    import torch
    xd = torch.from_numpy(x).cuda()
    yd = torch.from_numpy(y0.copy()).cuda()
    A.spmv(xd, yd)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


@pytest.mark.parametrize("s", [16, 32, 64, 128, 256])
@pytest.mark.parametrize("tile_nnz", [-1, 4, 0, 1000000])
def test_slice_spmv_is_the_reference_order(gpu, s, tile_nnz):
    for coo in cases():
        x = W.rhs(coo.n, 7)
        y0 = W.rhs(coo.m, 8)
        A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s,
                                      slice_tile_nnz=tile_nnz)
        np.testing.assert_array_equal(_spmv(A, x, y0), reference_y(coo, x, y0), err_msg=coo.name)
        assert A.device_status() == 0
        A.release()


@pytest.mark.parametrize("s", [16, 32, 64, 128, 256])
@pytest.mark.parametrize("tile_nnz", [4, 0, 1000000])
def test_slices_equal_the_oracle_encoding(gpu, s, tile_nnz):
    avg = DEFAULT_TILE_NNZ if tile_nnz == 0 else tile_nnz
    for coo in cases():
        A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s,
                                      slice_tile_nnz=tile_nnz)
        got = A.slices()
        b = oracle.build(coo.rows, coo.cols, coo.vals, coo.m, coo.n, s)
        ref = b.slices(avg)
        for k in ("slices", "slots", "lane_records", "elements", "block_rows"):
            assert got[k] == ref[k], (coo.name, k)
        for k in ("base", "meta", "brow", "steps", "lanes", "chain", "lane", "words"):
            np.testing.assert_array_equal(got[k], ref[k], err_msg=f"{coo.name} {k}")
        # values: the format's values in slot order, zero in the padding
        want = np.where(ref["vidx"] >= 0, b.values[np.maximum(ref["vidx"], 0)], 0).astype(b.values.dtype)
        np.testing.assert_array_equal(got["values"], want)
        A.release()


def test_chains_and_bitmap_tiles_are_exercised(gpu):
    """The cases above reach the paths they are there for: one-row chains and
    slice block rows that hold a bitmap tile."""
    coo = heavy_rows()
    P = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64).slices()
    assert P["chain"].sum() >= 4 and (P["steps"][P["chain"] == 1] > 256).all()
    coo = bitmap_in_sparse_rows()
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
    P = A.slices()
    e = A.export()
    bitmap_rows = {int(np.searchsorted(e["brow_ptr"], t, side="right") - 1)
                   for t in np.nonzero(e["tile_scheme"] == 2)[0]}
    served = set()  # block rows the slices sum: a chain's own, a sliced lane's row's
    for q in range(P["slices"]):
        if P["chain"][q]:
            served.add(int(P["brow"][q]))
        else:
            for l in range(int(P["lanes"][q])):
                served.add((int(P["brow"][q]) * 64 + int(P["lane"][P["meta"][q] + l] >> 8)) // 64)
    assert bitmap_rows and bitmap_rows <= served


@pytest.mark.parametrize("vt", ["f32", "bf16"])
@pytest.mark.parametrize("s", [16, 64, 256])
def test_slice_spmv_f32_bitwise_against_oracle(gpu, vt, s):
    """f32 / bf16 values through the slices; at block sizes 16 and 256 the
    slices serve these matrices alone (no dense tile)."""
    import torch
    for coo in (W.rmat(1 << 14, 8, seed=4), heavy_rows(seed=2)):
        A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, value_type=vt,
                                      slice_tile_nnz=1000000)
        assert A.slices()["slices"] > 0
        rng = np.random.default_rng(4)
        x32 = rng.uniform(-1, 1, coo.n).astype(np.float32)
        y32 = rng.standard_normal(coo.m).astype(np.float32)
        xd, yd = torch.from_numpy(x32).cuda(), torch.from_numpy(y32.copy()).cuda()
        A.spmv_f32(xd, yd)
        torch.cuda.synchronize()
        order = np.lexsort((coo.cols, coo.rows))
        v32 = oracle.values_as_f32(coo.vals[order], vt)
        ref = oracle.spmv_elements_f32(coo.rows[order], coo.cols[order], v32, x32, y32.copy())
        np.testing.assert_array_equal(yd.cpu().numpy(), ref)


def test_slice_spmm_columns_equal_their_spmv(gpu):
    import torch
    coo = heavy_rows(seed=3)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
    rng = np.random.default_rng(5)
    # passes of 32, 16, 8, 4, 2 and 1 columns through the sliced rows and the
    # chains; X and Y inside wider buffers (ldx = k + 3, ldy = k + 5)
    for k in (1, 2, 3, 8, 13, 16, 32, 63):
        Xb = torch.from_numpy(rng.uniform(-1, 1, (coo.n, k + 3))).cuda()
        Yb = torch.from_numpy(rng.standard_normal((coo.m, k + 5))).cuda()
        Yc = Yb.clone()
        X, Y = Xb[:, :k], Yc[:, :k]
        A.spmm(X, Y)
        assert torch.equal(Yc[:, k:], Yb[:, k:])  # nothing outside the k columns
        for j in range(k):
            y = Yb[:, j].contiguous()
            A.spmv(X[:, j].contiguous(), y)
            assert torch.equal(Y[:, j], y), (k, j)
    sl = A.slices()
    assert sl["chain"].sum() > 0 and (sl["chain"] == 0).sum() > 0  # both kernels ran


def test_slice_batch_equals_each_matrix_alone(gpu):
    import torch
    coos = [W.rmat(1 << 12, 8, seed=i) for i in range(6)] + [heavy_rows(seed=4), W.banded(3000, 5, seed=2)]
    mats = [AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=64) for c in coos]
    rng = np.random.default_rng(6)
    xs = [torch.from_numpy(rng.uniform(-1, 1, c.n)).cuda() for c in coos]
    ys = [torch.from_numpy(rng.standard_normal(c.m)).cuda() for c in coos]
    alone = []
    for A, x, y in zip(mats, xs, ys):
        yy = y.clone()
        A.spmv(x, yy)
        alone.append(yy)
    b = AbhsfBatch(mats)
    for _ in range(2):  # consecutive calls from the same inputs
        yb = [y.clone() for y in ys]
        b.spmv(xs, yb)
        torch.cuda.synchronize()
        for i, (p, q) in enumerate(zip(yb, alone)):
            assert torch.equal(p, q), i
    assert b.status() == 0
    b.release()


def test_slice_host_pipeline(gpu):
    """abhsf_spmv_host on a matrix of 2^20 rows (the chunked copy pipeline),
    its hypersparse block rows summed from slices chunk by chunk."""
    coo = W.rmat(1 << 20, 4, seed=9)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
    assert A.slices()["slices"] > 0
    x = W.rhs(coo.n, 1)
    y = W.rhs(coo.m, 2)
    ref = reference_y(coo, x, y)
    A.spmv(x, y)
    np.testing.assert_array_equal(y, ref)


def test_long_chains(gpu):
    """Rows of 40,000, 25,000 and 9,000 elements (chains: many full groups of
    256 products through the shared buffer, and a partial last group) over a
    hypersparse rest: FP64 SpMV (twice, from the same y), f32 SpMV and SpMM
    bitwise in the reference order."""
    import torch
    coo = heavy_rows(n=120000, heavy=(3, 777), per_heavy=40000, sparse=150000, seed=8)
    rng = np.random.default_rng(9)
    extra_r = np.concatenate([np.full(25000, 9001, np.int64), np.full(9000, 50000, np.int64)])
    extra_c = np.concatenate([rng.choice(coo.n, 25000, replace=False), rng.choice(coo.n, 9000, replace=False)])
    rows = np.concatenate([coo.rows[coo.rows != 777], extra_r])
    cols = np.concatenate([coo.cols[coo.rows != 777], extra_c])
    key = np.unique(rows * coo.n + cols)
    rows, cols = key // coo.n, key % coo.n
    vals = rng.standard_normal(rows.size)
    A = AbhsfMatrix.from_elements(rows, cols, vals, coo.n, coo.n, block_size=64)
    sl = A.slices()
    lens = sl["steps"][sl["chain"] == 1]
    big = sorted(lens[lens >= 16384].tolist())  # the rest adds a few elements to some heavy rows
    assert len(big) == 2 and 25000 <= big[0] < 25100 and 40000 <= big[1] < 40100
    assert ((lens >= 9000) & (lens < 9100)).sum() == 1
    assert A.kernels() == 2  # sliced rows, chains
    x = rng.uniform(-1, 1, coo.n)
    y0 = rng.standard_normal(coo.n)
    for _ in range(2):
        yd = torch.from_numpy(y0.copy()).cuda()
        A.spmv(torch.from_numpy(x).cuda(), yd)
        np.testing.assert_array_equal(yd.cpu().numpy(), oracle.spmv_elements(rows, cols, vals, x, y0.copy()))
    X = rng.uniform(-1, 1, (coo.n, 3))
    Y0 = rng.standard_normal((coo.n, 3))
    Y = torch.from_numpy(Y0.copy()).cuda()
    A.spmm(torch.from_numpy(X).cuda(), Y)
    for j in range(3):
        np.testing.assert_array_equal(Y[:, j].cpu().numpy(),
                                      oracle.spmv_elements(rows, cols, vals, X[:, j].copy(), Y0[:, j].copy()))
    A32 = AbhsfMatrix.from_elements(rows, cols, vals, coo.n, coo.n, block_size=64, value_type="f32")
    x32 = x.astype(np.float32)
    y32 = y0.astype(np.float32)
    yd = torch.from_numpy(y32.copy()).cuda()
    A32.spmv_f32(torch.from_numpy(x32).cuda(), yd)
    v32 = oracle.values_as_f32(vals, "f32")
    np.testing.assert_array_equal(yd.cpu().numpy(), oracle.spmv_elements_f32(rows, cols, v32, x32, y32.copy()))
