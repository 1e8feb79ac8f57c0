"""GPU f32 SpMV for matrices stored as f32 or bf16 (abhsf_spmv_f32): values
widened to f32, each product and each sum rounded to f32, per row in the
reference's column order, at every block size (the ring kernel at 32 and 64,
the streaming kernel at 16, 128 and 256 beside the row slices or alone).
Checked bitwise against the oracle's f32 loop over the stored values, and its
error against the FP64 product measured."""
import numpy as np
import pytest

from abhsf_b200 import AbhsfMatrix, capi
from abhsf_b200 import workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu


def _run_f32(A, x32, y32):
    import torch
    xd = torch.from_numpy(np.ascontiguousarray(x32)).cuda()
    yd = torch.from_numpy(np.array(y32, dtype=np.float32)).cuda()
    A.spmv_f32(xd, yd)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def _oracle_f32(coo, vt, x32, y32):
    order = np.lexsort((coo.cols, coo.rows))
    v32 = oracle.values_as_f32(coo.vals[order], vt)
    return oracle.spmv_elements_f32(coo.rows[order], coo.cols[order], v32, x32, y32)


@pytest.mark.parametrize("vt", ["f32", "bf16"])
@pytest.mark.parametrize("s", [32, 64])
@pytest.mark.parametrize("forced", [None, "coo", "csr", "bitmap", "dense"])
def test_spmv_f32_bitwise_against_oracle(gpu, vt, s, forced):
    coo = W.random_blocky(1900, 2300, s, 150, seed=21)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, value_type=vt,
                                  forced_scheme=forced)
    rng = np.random.default_rng(4)
    x32 = rng.uniform(-1, 1, coo.n).astype(np.float32)
    y32 = rng.standard_normal(coo.m).astype(np.float32)
    np.testing.assert_array_equal(_run_f32(A, x32, y32), _oracle_f32(coo, vt, x32, y32))
    assert A.device_status() == 0


@pytest.mark.parametrize("vt", ["f32", "bf16"])
@pytest.mark.parametrize("s", [16, 128, 256])
@pytest.mark.parametrize("slices", [True, False])
@pytest.mark.parametrize("forced", [None, "coo", "csr", "bitmap", "dense"])
def test_spmv_f32_streaming_sizes_bitwise(gpu, vt, s, slices, forced):
    """Block sizes without a ring kernel: the streaming kernel takes the block
    rows the row slices leave (all of them with slices switched off), over
    every scheme, with ragged edges (m, n not multiples of s)."""
    coo = W.random_blocky(1900, 2300, s, 150, seed=23)
    if forced == "csr" and s == 256:
        # a CSR tile holds at most 65535 elements: every 16th element out
        keep = np.arange(coo.rows.size) % 16 != 0
        coo = W.Coo(coo.rows[keep], coo.cols[keep], coo.vals[keep], coo.m, coo.n, coo.name)
    kw = {} if slices else {"slice_tile_nnz": -1}
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, value_type=vt,
                                  forced_scheme=forced, **kw)
    rng = np.random.default_rng(5)
    x32 = rng.uniform(-1, 1, coo.n).astype(np.float32)
    y32 = rng.standard_normal(coo.m).astype(np.float32)
    np.testing.assert_array_equal(_run_f32(A, x32, y32), _oracle_f32(coo, vt, x32, y32))
    assert A.device_status() == 0


@pytest.mark.parametrize("vt", ["f32", "bf16"])
@pytest.mark.parametrize("s", [16, 128])
def test_spmv_f32_power_law_beside_slices(gpu, vt, s):
    """R-MAT rows: hypersparse block rows in slices (long rows in chains),
    the dense ones in the streaming kernel, in one call."""
    coo = W.rmat(1 << 13, 12, seed=4)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, value_type=vt)
    x32 = np.random.default_rng(6).uniform(-1, 1, coo.n).astype(np.float32)
    y32 = np.zeros(coo.m, np.float32)
    np.testing.assert_array_equal(_run_f32(A, x32, y32), _oracle_f32(coo, vt, x32, y32))


@pytest.mark.parametrize("vt", ["f32", "bf16"])
def test_spmv_f32_laplacian_exact_values(gpu, vt):
    """3D Laplacian: 6 and -1 are exact in f32 and bf16, so only the f32
    arithmetic differs from FP64."""
    coo = W.laplacian_3d(20)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64, value_type=vt)
    x32 = np.random.default_rng(1).uniform(-1, 1, coo.n).astype(np.float32)
    y = _run_f32(A, x32, np.zeros(coo.m, np.float32))
    np.testing.assert_array_equal(y, _oracle_f32(coo, vt, x32, np.zeros(coo.m, np.float32)))


@pytest.mark.parametrize("vt,bound", [("f32", 2e-6), ("bf16", 2e-2)])
def test_spmv_f32_error_against_fp64(gpu, vt, bound):
    """Scaled error |y - y64| / (|A| |x|) per row stays within the storage
    precision (2^-24 for f32 values, 2^-9 for bf16) times a small factor."""
    coo = W.random_blocky(3000, 3000, 64, 200, seed=9)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64, value_type=vt)
    x32 = np.random.default_rng(2).uniform(-1, 1, coo.n).astype(np.float32)
    y = _run_f32(A, x32, np.zeros(coo.m, np.float32)).astype(np.float64)
    x64 = x32.astype(np.float64)
    y64 = oracle.spmv_elements(coo.rows, coo.cols, coo.vals, x64, np.zeros(coo.m))
    scale = oracle.abs_spmv(coo.rows, coo.cols, coo.vals, x64, coo.m)
    nz = scale > 0
    assert np.max(np.abs(y - y64)[nz] / scale[nz]) <= bound


def test_spmv_f32_arguments(gpu):
    import torch
    coo = W.random_blocky(300, 200, 64, 10, seed=1)
    A64 = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n)
    x = torch.zeros(200, dtype=torch.float32, device="cuda")
    y = torch.zeros(300, dtype=torch.float32, device="cuda")
    assert capi.lib.abhsf_spmv_f32(A64.handle, x.data_ptr(), y.data_ptr(), None) == capi.INVALID_VALUE
    # block size 16 with no row slices: the streaming kernel alone
    A16 = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=16, value_type="f32",
                                    slice_tile_nnz=-1)
    assert capi.lib.abhsf_spmv_f32(A16.handle, x.data_ptr(), y.data_ptr(), None) == capi.SUCCESS
    torch.cuda.synchronize()
    assert not torch.any(torch.isnan(y))
    assert capi.lib.abhsf_spmv_f32(A16.handle, None, y.data_ptr(), None) == capi.INVALID_VALUE
