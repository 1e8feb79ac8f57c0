"""The reference's per-scheme block benchmark matrix (block_generator and
main of spmv/orig/88.cpp): num_blocks^2 copies of one 8 x 8 block pattern,
values 1.0, x = 1.  Its known answer, the "y-vector sum" the reference prints
(88.cpp:823-828), is (iterations) * bnnz * num_blocks^2 whatever the pattern:
checked on the oracle here, and on the GPU for every scheme the tiles take
(at s = 64 a tile holds 64 blocks: bnnz 1 -> COO, 4 -> CSR, 16 -> bitmap,
64 -> dense)."""
import numpy as np
import pytest

from abhsf_b200 import workloads as W
from oracle import oracle

# 88.cpp:40-41: 40 timed + 5 warm-up products into a y that is not reset
REF_ITERATIONS = 40 + 5


@pytest.mark.parametrize("bnnz", [1, 2, 4, 8, 16, 32, 64])
def test_random_pattern_is_bnnz_distinct_positions_in_row_order(bnnz):
    p = W.block_pattern(bnnz)
    assert p.shape == (bnnz, 2)
    assert len({tuple(q) for q in p.tolist()}) == bnnz
    assert p.min() >= 0 and p.max() < 8
    assert np.all(np.diff(p[:, 0] * 8 + p[:, 1]) > 0)  # std::set order, walked row-major by finalize
    np.testing.assert_array_equal(W.block_pattern(bnnz), p)  # seeded
    if bnnz == 64:
        np.testing.assert_array_equal(p[:, 0] * 8 + p[:, 1], np.arange(64))


def test_fixed_patterns_and_argument_checks():
    np.testing.assert_array_equal(W.block_pattern(kind="diagonal"), np.stack([np.arange(8)] * 2, 1))
    np.testing.assert_array_equal(W.block_pattern(kind="single_row"), np.stack([np.zeros(8, int), np.arange(8)], 1))
    np.testing.assert_array_equal(W.block_pattern(kind="single_col"), np.stack([np.arange(8), np.zeros(8, int)], 1))
    for bad in (0, 65):
        with pytest.raises(ValueError):
            W.block_pattern(bad)
    with pytest.raises(ValueError):
        W.block_pattern(kind="checkerboard")


@pytest.mark.parametrize("kind,bnnz", [("random", 1), ("random", 13), ("random", 64), ("diagonal", 8),
                                       ("single_row", 8), ("single_col", 8)])
def test_every_block_is_the_pattern_and_the_known_sum_holds(kind, bnnz):
    nb = 24
    coo = W.identical_blocks(nb, bnnz, kind)
    pat = W.block_pattern(bnnz, kind)
    assert (coo.m, coo.n, coo.nnz) == (8 * nb, 8 * nb, nb * nb * pat.shape[0])
    assert np.all(coo.vals == 1.0)
    keys = coo.rows * coo.n + coo.cols
    assert np.all(np.diff(keys) > 0)  # row order, no duplicates
    local = set(zip((coo.rows % 8).tolist(), (coo.cols % 8).tolist()))
    assert local == {tuple(q) for q in pat.tolist()}
    per_block = np.bincount((coo.rows // 8) * nb + coo.cols // 8, minlength=nb * nb)
    assert np.all(per_block == pat.shape[0])
    x = np.ones(coo.n)
    y = np.zeros(coo.m)
    for _ in range(REF_ITERATIONS):
        oracle.spmv_elements(coo.rows, coo.cols, coo.vals, x, y)
    assert y.sum() == REF_ITERATIONS * pat.shape[0] * nb * nb
    row_counts = np.bincount(pat[:, 0], minlength=8)
    np.testing.assert_array_equal(y, REF_ITERATIONS * nb * row_counts[np.arange(coo.m) % 8])


@pytest.mark.gpu
@pytest.mark.parametrize("s", [32, 64])
@pytest.mark.parametrize("kind,bnnz", [("random", 1), ("random", 4), ("random", 16), ("random", 64),
                                       ("diagonal", 8), ("single_row", 8), ("single_col", 8)])
def test_gpu_known_sum_and_oracle_bits(gpu, s, kind, bnnz):
    import torch

    from abhsf_b200 import AbhsfMatrix
    nb = 128
    coo = W.identical_blocks(nb, bnnz, kind)
    z = W.block_pattern(bnnz, kind).shape[0]
    A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=s)
    per_tile = z * (s // 8) ** 2
    st = A.stats()
    want_scheme = oracle.select_scheme(s, s, per_tile, 64)
    assert st["tiles"] == (coo.m // s) ** 2
    assert st["tiles_per_scheme"][("coo", "csr", "bitmap", "dense")[want_scheme]] == st["tiles"]
    x = torch.ones(coo.n, dtype=torch.float64, device="cuda")
    y = torch.zeros(coo.m, dtype=torch.float64, device="cuda")
    k = 5
    for _ in range(k):
        A.spmv(x, y)
    torch.cuda.synchronize()
    got = y.cpu().numpy()
    want = np.zeros(coo.m)
    for _ in range(k):
        oracle.spmv_elements(coo.rows, coo.cols, coo.vals, np.ones(coo.n), want)
    np.testing.assert_array_equal(got, want)
    assert got.sum() == k * z * nb * nb
    assert A.device_status() == 0
    A.release()
