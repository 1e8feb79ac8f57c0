"""GPU SpMV parity: y += A x on the B200 against the FP64 oracle (the
reference's verification loop) and the reference CSR spmv_naive (golden),
with non-unit random values and x so that order and placement errors show."""
import numpy as np
import pytest

from conftest import assert_spmv_close, golden_matrices, golden_spmv, golden_stats
from abhsf_b200 import AbhsfMatrix, capi
from abhsf_b200 import workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu

MATS = golden_matrices()
STATS = golden_stats()


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run_spmv(A, x, y0):
    import torch
    xd, yd = _dev(x), _dev(y0.copy())
    A.spmv(xd, yd)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def reference_order_y(coo, x, y0):
    """The reference CSR's y: products added one at a time per row, columns
    ascending (the oracle loop on row-major sorted elements reproduces the
    reference's spmv_naive bit for bit, tests/test_oracle_golden.py)."""
    order = np.lexsort((coo.cols, coo.rows))
    return oracle.spmv_elements(coo.rows[order], coo.cols[order], coo.vals[order], x, y0.copy())


def check_y(order, y, coo, x, y0):
    if order == "reference":
        np.testing.assert_array_equal(y, reference_order_y(coo, x, y0))
    else:
        ref = oracle.spmv_elements(coo.rows, coo.cols, coo.vals, x, y0.copy())
        scale = oracle.abs_spmv(coo.rows, coo.cols, coo.vals, x, coo.m) + np.abs(y0)
        assert_spmv_close(y, ref, scale)


@pytest.mark.parametrize("order", ["reference", "tree"])
@pytest.mark.parametrize("s", [16, 32, 64, 128, 256])
@pytest.mark.parametrize("forced", [None, "coo", "csr", "bitmap", "dense"])
def test_spmv_matches_oracle_all_schemes(gpu, s, forced, order):
    for name, coo in MATS.items():
        x = W.rhs(coo.n, 11)
        y0 = W.rhs(coo.m, 12)
        A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, forced_scheme=forced,
                                      sum_order=order)
        check_y(order, run_spmv(A, x, y0), coo, x, y0)
        assert A.device_status() == 0
        A.release()


@pytest.mark.parametrize("order", ["reference", "tree"])
def test_spmv_matches_reference_csr_golden(gpu, order):
    ref = golden_spmv()
    n_checked = 0
    for name, coo in MATS.items():
        if name + "__y" not in ref:
            continue
        x, y0, yr = ref[name + "__x"], ref[name + "__y0"], ref[name + "__y"]
        scale = oracle.abs_spmv(coo.rows, coo.cols, coo.vals, x, coo.m) + np.abs(y0)
        for s in (16, 64, 256):
            A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, sum_order=order)
            y = run_spmv(A, x, y0)
            if order == "reference":
                np.testing.assert_array_equal(y, yr, err_msg=f"{name} s={s}")
            else:
                assert_spmv_close(y, yr, scale)
            A.release()
        n_checked += 1
    assert n_checked >= 6


@pytest.mark.parametrize("order", ["reference", "tree"])
def test_spmv_laplace2d_512_against_golden(gpu, order):
    c = W.laplacian_2d(512)
    x = W.rhs(c.n, 0)
    yr = golden_spmv()["laplace2d_512__y_seed0"]
    A = AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=64, sum_order=order)
    y = run_spmv(A, x, np.zeros(c.m))
    scale = oracle.abs_spmv(c.rows, c.cols, c.vals, x, c.m)
    worst_scaled, worst_rel = assert_spmv_close(y, yr, scale)
    if order == "reference":
        # bitwise the reference CSR's y: 0 relative error on every element
        np.testing.assert_array_equal(y, yr)
    else:
        # tree-ordered sums: the scaled bound holds; |dy|/|y| alone is order
        # dependent on rows that cancel (4 x_i minus four neighbours)
        assert worst_scaled <= 1e-13, worst_scaled


def test_wait_timeout_sets_status_and_context_survives(gpu):
    """A copy wait that runs out (the bulk copies of one tile are never
    issued) ends the kernel with ABHSF_DEVSTAT_WAIT_TIMEOUT instead of hanging;
    the context and the matrix stay usable."""
    import torch
    coo = W.random_blocky(2000, 2000, 64, 300, seed=31)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64, slice_tile_nnz=-1)
    x = W.rhs(coo.n, 1)
    y0 = np.zeros(coo.m)
    try:
        capi.lib.abhsf_test_set_hooks(2, 1 << 12)
        run_spmv(A, x, y0)
        st = A.device_status(clear=True)
    finally:
        capi.lib.abhsf_test_set_hooks(-1, 0)
    assert st & capi.DEVSTAT_WAIT_TIMEOUT
    y = run_spmv(A, x, y0)
    assert A.device_status() == 0
    np.testing.assert_array_equal(y, reference_order_y(coo, x, y0))
    torch.cuda.synchronize()


def test_host_pointer_path_equals_device_path(gpu):
    coo = MATS["blocky64"]
    x = W.rhs(coo.n, 3)
    y0 = W.rhs(coo.m, 4)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
    yh = y0.copy()
    A.spmv(x, yh)  # numpy: host buffers, copies inside the call
    yd = run_spmv(A, x, y0)
    np.testing.assert_array_equal(yh, yd)


@pytest.mark.parametrize("s", [32, 64])
def test_pipelined_host_path_equals_device_path(gpu, s):
    """Host-memory x and y of a matrix with at least 2^20 rows go through the
    chunked pipeline (y copied in and out chunk by chunk around one kernel
    launch per chunk of block rows): y is bitwise the device path's, on
    consecutive calls, with empty and non-empty chunks."""
    import torch
    n = (1 << 20) + 37
    band = W.banded(n, 3, seed=5)
    M = -(-n // s)  # block rows; the second of the pipeline's four chunks, [M/4, M/2), left empty
    keep = (band.rows < (M // 4) * s) | (band.rows >= (M // 2) * s)
    cases = [W.Coo(band.rows[keep], band.cols[keep], band.vals[keep], n, n, "band_gap"),
             W.tiled_mixture(n=n, p=2e-5, seed=6)]
    for coo in cases:
        x = W.rhs(coo.n, 5)
        y0 = W.rhs(coo.m, 6)
        A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s)
        want = run_spmv(A, x, y0)
        x_pin = torch.from_numpy(x).pin_memory().numpy()
        for _ in range(2):
            yh = torch.from_numpy(y0.copy()).pin_memory().numpy()
            A.spmv(x_pin, yh)
            np.testing.assert_array_equal(yh, want, err_msg=coo.name)
        yp = y0.copy()  # pageable host memory works too
        A.spmv(x, yp)
        np.testing.assert_array_equal(yp, want, err_msg=coo.name)
        assert A.device_status() == 0
        A.release()


@pytest.mark.parametrize("order", ["reference", "tree"])
def test_spmv_is_deterministic(gpu, order):
    coo = W.random_blocky(3000, 3000, 64, 400, seed=21)
    x = W.rhs(coo.n, 5)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64, sum_order=order)
    ys = [run_spmv(A, x, np.zeros(coo.m)) for _ in range(3)]
    np.testing.assert_array_equal(ys[0], ys[1])
    np.testing.assert_array_equal(ys[0], ys[2])


def test_spmv_argument_errors(gpu):
    import torch
    coo = MATS["rand_real"]
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=32)
    with pytest.raises(capi.InvalidValue):
        A.spmv(torch.zeros(coo.n, device="cuda"), torch.zeros(coo.m, device="cuda"))  # float32
    with pytest.raises(capi.InvalidValue):
        A.spmv(torch.zeros(coo.n + 1, dtype=torch.float64, device="cuda"),
               torch.zeros(coo.m, dtype=torch.float64, device="cuda"))
    B = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=32, value_type="f32")
    with pytest.raises(capi.InvalidValue):
        B.spmv(torch.zeros(coo.n, dtype=torch.float64, device="cuda"),
               torch.zeros(coo.m, dtype=torch.float64, device="cuda"))
    A.release()
    with pytest.raises(capi.InvalidValue):
        A.spmv(np.zeros(coo.n), np.zeros(coo.m))


def test_device_inputs_build(gpu):
    coo = MATS["blocky16"]
    A = AbhsfMatrix.from_elements(_dev(coo.rows), _dev(coo.cols), _dev(coo.vals), coo.m, coo.n, block_size=16)
    B = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=16)
    ea, eb = A.export(), B.export()
    for k in ea:
        np.testing.assert_array_equal(ea[k], eb[k])


@pytest.mark.parametrize("s", [64])
def test_tiled_mixture_full_size(gpu, s):
    """The throughput workload at full size (n = 4,194,304, ~60M nnz): format
    statistics against the oracle histogram and the cost model; y bitwise
    against the reference CSR (reference order) and within the bound against
    the FP64 oracle loop (tree order)."""
    c = W.tiled_mixture()
    assert 50_000_000 < c.nnz < 70_000_000
    A = AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=s)
    B = AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=s, sum_order="tree")
    st = A.stats()
    hist = oracle.block_histogram(c.rows, c.cols, 6, 6)
    assert st["tiles"] == sum(hist.values())
    want = {k: 0 for k in capi.SCHEME_NAMES}
    for z, cnt in hist.items():
        want[capi.SCHEME_NAMES[oracle.select_scheme(64, 64, z, 64)]] += cnt
    assert st["tiles_per_scheme"] == want
    x = W.rhs(c.n, 1)
    y0 = W.rhs(c.m, 2)
    ref = oracle.spmv_elements(c.rows, c.cols, c.vals, x, y0.copy())
    scale = oracle.abs_spmv(c.rows, c.cols, c.vals, x, c.m) + np.abs(y0)
    assert_spmv_close(run_spmv(B, x, y0), ref, scale)
    if oracle.RefCSR.available():
        yr = y0.copy()
        R = oracle.RefCSR(c.rows, c.cols, c.vals, c.m, c.n)
        R.spmv(x, yr)
        R.release()
    else:
        yr = reference_order_y(c, x, y0)
    np.testing.assert_array_equal(run_spmv(A, x, y0), yr)


def test_tiled_mixture_medium_every_row(gpu):
    """n = 1,048,576: many block rows made of one small COO tile (most of
    whose rows have no element) next to bitmap-heavy ones; every row,
    including the untouched ones, bitwise in the reference order."""
    c = W.tiled_mixture(n=1048576)
    A = AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=64)
    x = np.random.default_rng(3).uniform(-1, 1, c.n)
    y0 = np.random.default_rng(4).standard_normal(c.m)
    np.testing.assert_array_equal(run_spmv(A, x, y0), reference_order_y(c, x, y0))


@pytest.mark.parametrize("s", [32, 64])
def test_every_ring_variant_gives_the_reference_y(gpu, s):
    """The ring kernel's launch variants (consumer layouts: one or two teams
    of s/32 warps, four or two teams of one warp with s/32 rows per lane; x / y
    blocks as bulk copies or element copies) that the build times and chooses
    among give the reference CSR's y bit for bit, on matrices of few large
    tiles, of many small tiles (a 3D stencil) and with ragged edges (every
    block row on the ring: no row slices)."""
    import ctypes as C
    cases = [W.random_blocky(2100, 1900, s, 60, seed=3), W.laplacian_3d(20), W.rmat(3000, 8, seed=4),
             W.tiled_mixture(n=65536 + 37, p=1e-3, seed=2)]
    for coo in cases:
        x = W.rhs(coo.n, 21)
        y0 = W.rhs(coo.m, 22)
        want = reference_order_y(coo, x, y0)
        A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, slice_tile_nnz=-1)
        t, b = C.c_int32(), C.c_int32()
        assert capi.lib.abhsf_test_ring_variant(A.handle, 0, C.byref(t), C.byref(b)) == capi.SUCCESS
        assert t.value in (0, 1, 2, 3) and b.value in (0, 1)
        for layout in (0, 1, 2, 3):
            for bulk in (0, 1):
                t.value, b.value = layout, bulk
                assert capi.lib.abhsf_test_ring_variant(A.handle, 1, C.byref(t), C.byref(b)) == capi.SUCCESS
                np.testing.assert_array_equal(run_spmv(A, x, y0), want, err_msg=f"{coo.name} {layout} {bulk}")
        assert A.device_status() == 0
        A.release()


def test_ring_variant_environment_override(gpu, monkeypatch):
    """ABHSF_RING_VARIANT fixes the launch variant the build would time;
    malformed values fall back to timing."""
    import ctypes as C
    coo = W.laplacian_3d(12)
    t, b = C.c_int32(), C.c_int32()
    for value, want in (("2,0", (2, 0)), ("3,1", (3, 1))):
        monkeypatch.setenv("ABHSF_RING_VARIANT", value)
        A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64, slice_tile_nnz=-1)
        assert capi.lib.abhsf_test_ring_variant(A.handle, 0, C.byref(t), C.byref(b)) == capi.SUCCESS
        assert (t.value, b.value) == want
        A.release()
    monkeypatch.setenv("ABHSF_RING_VARIANT", "7,1")
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64, slice_tile_nnz=-1)
    assert capi.lib.abhsf_test_ring_variant(A.handle, 0, C.byref(t), C.byref(b)) == capi.SUCCESS
    assert t.value in (0, 1, 2, 3)
    x, y0 = W.rhs(coo.n, 1), W.rhs(coo.m, 2)
    np.testing.assert_array_equal(run_spmv(A, x, y0), reference_order_y(coo, x, y0))
    A.release()
