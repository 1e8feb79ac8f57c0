"""GPU conjugate gradients: plain FP64 CG and FP64 iterative refinement
around an f32 CG on an f32 / bf16 copy of the matrix.  The residual each
solver reports is checked against one computed on the CPU from the returned
x with the FP64 matrix."""
import numpy as np
import pytest

from abhsf_b200 import AbhsfMatrix, capi, cg, cg_mixed
from abhsf_b200 import workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu


def _cpu_rel_residual(coo, b, x):
    ax = oracle.spmv_elements(coo.rows, coo.cols, coo.vals, x, np.zeros(coo.m))
    return np.linalg.norm(b - ax) / np.linalg.norm(b)


def _vectors(n, seed):
    import torch
    b = np.random.default_rng(seed).uniform(-1, 1, n)
    return b, torch.from_numpy(b).cuda(), torch.zeros(n, dtype=torch.float64, device="cuda")


def _shifted_laplacian_2d(g, shift, seed):
    """2D Laplacian plus a random positive diagonal: SPD, well conditioned,
    values not representable in bf16."""
    coo = W.laplacian_2d(g)
    vals = coo.vals.copy()
    diag = coo.rows == coo.cols
    vals[diag] += shift * (1.0 + np.random.default_rng(seed).uniform(0, 1, int(diag.sum())))
    return W.Coo(coo.rows, coo.cols, vals, coo.m, coo.n)


@pytest.mark.parametrize("offset", [0, 1])
def test_cg_unaligned_and_odd_length_vectors(gpu, offset):
    """x and b 8 bytes past a 16-byte boundary (the vector kernels then take
    their element-by-element path) and n not a multiple of the 16-byte packs:
    the same solve, to the same residual, either way."""
    import torch
    coo = W.laplacian_3d(17)  # n = 4913, odd
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
    b = np.random.default_rng(3).uniform(-1, 1, coo.n)
    bb = torch.zeros(coo.n + 1, dtype=torch.float64, device="cuda")
    xb = torch.zeros(coo.n + 1, dtype=torch.float64, device="cuda")
    bd, xd = bb[offset:offset + coo.n], xb[offset:offset + coo.n]
    bd.copy_(torch.from_numpy(b))
    info = cg(A, bd, xd, rtol=1e-10)
    assert info["converged"]
    r = _cpu_rel_residual(coo, b, xd.cpu().numpy())
    assert r <= 1e-10 and abs(r - info["rel_residual"]) <= 1e-12
    A32 = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64, value_type="f32")
    xd.zero_()
    info = cg_mixed(A, A32, bd, xd, rtol=1e-10)
    assert info["converged"] and _cpu_rel_residual(coo, b, xd.cpu().numpy()) <= 1e-10


@pytest.mark.parametrize("s", [16, 64])
def test_cg_fp64_laplacian_3d(gpu, s):
    coo = W.laplacian_3d(24)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s)
    b, bd, xd = _vectors(coo.n, 1)
    info = cg(A, bd, xd, rtol=1e-10)
    assert info["converged"] and info["outer_iterations"] == 1 and info["iterations"] > 10
    r = _cpu_rel_residual(coo, b, xd.cpu().numpy())
    assert r <= 1e-10 and abs(r - info["rel_residual"]) <= 1e-12


@pytest.mark.parametrize("vt", ["f32", "bf16"])
@pytest.mark.parametrize("s", [16, 64, 128])
def test_cg_mixed_laplacian_3d_reaches_fp64_tolerance(gpu, vt, s):
    coo = W.laplacian_3d(24)
    A64 = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
    Alo = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s, value_type=vt)
    b, bd, xd = _vectors(coo.n, 2)
    info = cg_mixed(A64, Alo, bd, xd, rtol=1e-10)
    assert info["converged"] and info["outer_iterations"] >= 2
    r = _cpu_rel_residual(coo, b, xd.cpu().numpy())
    assert r <= 1e-10 and abs(r - info["rel_residual"]) <= 1e-12


@pytest.mark.parametrize("vt", ["f32", "bf16"])
def test_cg_mixed_inexact_low_precision_values(gpu, vt):
    """Values that the f32 / bf16 copy rounds: the refinement still reaches
    the FP64 tolerance because residuals use the FP64 matrix."""
    coo = _shifted_laplacian_2d(40, 2.0, 3)
    A64 = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=32)
    Alo = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=32, value_type=vt)
    b, bd, xd = _vectors(coo.n, 4)
    info = cg_mixed(A64, Alo, bd, xd, rtol=1e-11)
    assert info["converged"]
    assert _cpu_rel_residual(coo, b, xd.cpu().numpy()) <= 1e-11


def test_cg_iteration_limit_and_warm_start(gpu):
    coo = W.laplacian_3d(16)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n)
    b, bd, xd = _vectors(coo.n, 5)
    info = cg(A, bd, xd, rtol=1e-12, max_iters=5)
    assert not info["converged"] and 5 <= info["iterations"] < 5 + 8
    first = info["rel_residual"]
    info2 = cg(A, bd, xd, rtol=1e-10)  # continues from x
    assert info2["converged"] and info2["rel_residual"] < first


def test_cg_arguments(gpu):
    import torch
    coo = W.random_blocky(300, 200, 64, 10, seed=1)
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n)
    b = torch.zeros(200, dtype=torch.float64, device="cuda")
    info = capi.CgInfo()
    import ctypes as C
    assert capi.lib.abhsf_cg(A.handle, b.data_ptr(), b.data_ptr(), 1e-8, 10, C.byref(info), None) == \
        capi.INVALID_VALUE  # not square
