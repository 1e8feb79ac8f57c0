"""GPU batches: y_i += A_i x_i for many matrices in one launch
(abhsf_batch_spmv; the ring kernel at block sizes 32 and 64, the streaming
kernel at 16, 128 and 256, the slices beside either).  Every y_i must be bitwise what abhsf_spmv gives for that
matrix alone (the reference order), on consecutive calls, and when the launch
is captured in a CUDA graph and replayed."""
import ctypes as C

import numpy as np
import pytest

from abhsf_b200 import AbhsfBatch, AbhsfMatrix, capi
from abhsf_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _mixed_set(s):
    mats = [
        W.banded(3000, 7, seed=1),
        W.rmat(5000, 8, seed=2),
        W.random_blocky(2100, 1900, s, 60, seed=3),
        W.laplacian_2d(60),
        W.banded(64, 3, seed=4),
        W.Coo(np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0), 700, 500, "empty"),
        W.rmat(1000, 8, seed=5),
        W.Coo(np.array([0], np.int64), np.array([0], np.int64), np.array([2.5]), 1, 1, "one"),
        W.random_uniform(777, 1333, 20000, seed=6),
        W.banded(20000, 40, seed=7),
    ]
    return mats


def _vectors(coos, seed):
    import torch
    rng = np.random.default_rng(seed)
    xs = [torch.from_numpy(rng.uniform(-1, 1, c.n)).cuda() for c in coos]
    ys = [torch.from_numpy(rng.standard_normal(c.m)).cuda() for c in coos]
    return xs, ys


def _alone(A, x, y):
    import torch
    yy = y.clone()
    A.spmv(x, yy)
    torch.cuda.synchronize()
    return yy.cpu().numpy()


@pytest.mark.parametrize("s", [16, 32, 64, 128, 256])
def test_batch_equals_each_matrix_alone_on_consecutive_calls(gpu, s):
    import torch
    coos = _mixed_set(s)
    mats = [AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=s) for c in coos]
    batch = AbhsfBatch(mats)
    xs, ys = _vectors(coos, 1)
    want = [_alone(A, x, y) for A, x, y in zip(mats, xs, ys)]
    for _ in range(2):
        batch.spmv(xs, ys)
        torch.cuda.synchronize()
        for i, (y, w) in enumerate(zip(ys, want)):
            np.testing.assert_array_equal(y.cpu().numpy(), w, err_msg=f"matrix {i}")
        want = [_alone(A, x, y) for A, x, y in zip(mats, xs, ys)]
    assert batch.status() == 0


def test_batch_in_a_cuda_graph(gpu):
    import torch
    coos = _mixed_set(64)
    mats = [AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n) for c in coos]
    batch = AbhsfBatch(mats)
    xs, ys = _vectors(coos, 2)
    y0 = [y.clone() for y in ys]
    px, py = batch.pointer_tables(xs, ys)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        batch.spmv_tables(px, py, stream=s)  # warm-up outside the capture
    torch.cuda.synchronize()
    for y, y00 in zip(ys, y0):
        y.copy_(y00)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        batch.spmv_tables(px, py, stream=s)
    for y, y00 in zip(ys, y0):
        y.copy_(y00)
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    for A, x, y, y00 in zip(mats, xs, ys, y0):
        want = _alone(A, x, torch.from_numpy(_alone(A, x, y00)).cuda())  # two SpMVs
        np.testing.assert_array_equal(y.cpu().numpy(), want)


def test_batch_arguments(gpu):
    c = W.random_blocky(300, 200, 64, 10, seed=1)
    a64 = AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=64)
    a32 = AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=32)
    a16 = AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=16)
    f32 = AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=64, value_type="f32")
    h = C.c_void_p()

    def create(ms):
        arr = (C.c_void_p * len(ms))(*[m.handle for m in ms])
        return capi.lib.abhsf_batch_create(arr, len(ms), None, C.byref(h))

    assert create([a64, a32]) == capi.INVALID_VALUE
    assert create([a64, f32]) == capi.INVALID_VALUE
    assert create([a16, a16]) == capi.SUCCESS  # block size 16: the streaming kernel, one launch
    k = C.c_int32()
    assert capi.lib.abhsf_batch_kernels(h, C.byref(k)) == capi.SUCCESS and k.value >= 1
    assert capi.lib.abhsf_batch_release(h) == capi.SUCCESS
    assert capi.lib.abhsf_batch_create(None, 0, None, C.byref(h)) == capi.INVALID_VALUE
    assert create([a64, a64]) == capi.SUCCESS  # the same matrix twice is allowed
    assert capi.lib.abhsf_batch_spmv(h, None, None, None) == capi.INVALID_VALUE
    assert capi.lib.abhsf_batch_release(h) == capi.SUCCESS
