"""Parity at the benchmark sizes, bitwise against the reference's own CSR
spmv_naive (spmv/bottlenecks/spmv.cpp:58-64, compiled from the reference
sources into oracle/_ref; where that library is absent, the oracle's
element loop over row-major elements, which reproduces it bit for bit):

* R-MAT scale 22 (n = 4,194,304, edge factor 16, values N(0,1)), FP64, the
  default build (its hypersparse block rows in row slices and chains);
* every y_i of the 256-matrix batch in one batched launch;
* the tiled mixture at full size (n = 4,194,304, ~60M nonzeros) at block
  sizes 16, 128 and 256 (the streaming kernel beside the row slices).
"""
import numpy as np
import pytest

from abhsf_b200 import AbhsfBatch, AbhsfMatrix
from abhsf_b200 import workloads as W
from oracle import oracle

pytestmark = pytest.mark.gpu


def reference_y(rows, cols, vals, m, n, x, y0):
    y = y0.copy()
    if oracle.RefCSR.available():
        R = oracle.RefCSR(rows, cols, vals, m, n)
        R.spmv(x, y)
        R.release()
        return y
    order = np.lexsort((cols, rows))
    return oracle.spmv_elements(rows[order], cols[order], vals[order], x, y)


def _gpu_spmv(A, x, y0):
    import torch
    xd = torch.from_numpy(x).cuda()
    yd = torch.from_numpy(y0.copy()).cuda()
    A.spmv(xd, yd)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def test_rmat_scale22_fp64_bitwise(gpu):
    import torch
    rows, cols, vals, n = W.rmat_device(22, 16, seed=1, device="cuda")
    A = AbhsfMatrix.from_elements(rows, cols, vals, n, n, block_size=64)
    assert A.slices()["slices"] > 0
    r, c, v = rows.cpu().numpy(), cols.cpu().numpy(), vals.cpu().numpy()
    del rows, cols, vals
    torch.cuda.empty_cache()
    x = W.rhs(n, 5)
    y0 = W.rhs(n, 6)
    np.testing.assert_array_equal(_gpu_spmv(A, x, y0), reference_y(r, c, v, n, n, x, y0))
    assert A.device_status() == 0


def test_batch_of_256_every_y_bitwise(gpu):
    import torch
    coos, mats = [], []
    for rows, cols, vals, m, n, _ in W.batched_set_device(256, seed=0, device="cuda"):
        mats.append(AbhsfMatrix.from_elements(rows, cols, vals, m, n, block_size=64))
        coos.append((rows.cpu().numpy(), cols.cpu().numpy(), vals.cpu().numpy(), m, n))
    rng = np.random.default_rng(7)
    xs = [rng.uniform(-1, 1, c[4]) for c in coos]
    ys = [rng.standard_normal(c[3]) for c in coos]
    b = AbhsfBatch(mats)
    xd = [torch.from_numpy(x).cuda() for x in xs]
    yd = [torch.from_numpy(y.copy()).cuda() for y in ys]
    b.spmv(xd, yd)
    torch.cuda.synchronize()
    assert b.status() == 0
    for i, (c, x, y) in enumerate(zip(coos, xs, ys)):
        np.testing.assert_array_equal(yd[i].cpu().numpy(), reference_y(*c, x, y), err_msg=f"matrix {i}")


@pytest.mark.parametrize("s", [16, 128, 256])
def test_tiled_mixture_full_size_other_block_sizes(gpu, s):
    c = W.tiled_mixture()
    A = AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=s)
    x = W.rhs(c.n, 1)
    y0 = W.rhs(c.m, 2)
    np.testing.assert_array_equal(_gpu_spmv(A, x, y0), reference_y(c.rows, c.cols, c.vals, c.m, c.n, x, y0))
    assert A.device_status() == 0
