"""The oracle's restatement of the delta-coded row slices (orc_slices_build,
orc_spmv_slices), checked on the CPU: y through the slices is bitwise the
reference CSR order's y, and the encoding keeps the rules the library's SpMV
relies on -- every element at exactly one slot, each row's columns ascending,
sliced rows grouped by length within a segment of block rows (the quarters
of the block rows the host-memory SpMV works through one after another),
chains of more than 256 elements on their own.  The GPU encoding is tested
equal to this one word for word (tests/test_gpu_slices.py)."""
import numpy as np
import pytest

from abhsf_b200 import workloads as W
from oracle import oracle


def heavy_rows(n=20000, heavy=(0, 1, 5, 700), per_heavy=600, sparse=30000, seed=0) -> W.Coo:
    rng = np.random.default_rng(seed)
    r = [np.full(per_heavy, h, np.int64) for h in heavy]
    c = [rng.choice(n, per_heavy, replace=False) for _ in heavy]
    r.append(rng.integers(0, n, sparse))
    c.append(rng.integers(0, n, sparse))
    rows, cols = np.concatenate(r), np.concatenate(c)
    key = np.unique(rows * n + cols)
    rows, cols = key // n, key % n
    return W.Coo(rows, cols, rng.standard_normal(rows.size), n, n, "heavy_rows")


def cases():
    return [W.rmat(1 << 12, 8, seed=3), heavy_rows(), W.random_uniform(3000, 4000, 9000, seed=5),
            W.banded(2000, 3, seed=1)]


def segments(M):
    b = [0]
    for c in range(1, 5):
        e = M * c // 4
        if e > b[-1]:
            b.append(e)
    return b


@pytest.mark.parametrize("s", [16, 64, 256])
def test_oracle_slices_spmv_is_the_reference_order(s):
    for coo in cases():
        b = oracle.build(coo.rows, coo.cols, coo.vals, coo.m, coo.n, s)
        P = b.slices(1e9)
        if P["block_rows"] * s < coo.m // 2:
            continue  # dense tiles keep most rows away from the slices
        x = W.rhs(coo.n, 7)
        y0 = W.rhs(coo.m, 8)
        order = np.lexsort((coo.cols, coo.rows))
        ref = oracle.spmv_elements(coo.rows[order], coo.cols[order], coo.vals[order], x, y0.copy())
        y = y0.copy()
        b.spmv_slices(1e9, x, y)
        # the rows the slices serve: those of the slice block rows
        rows = set()
        for q in range(P["slices"]):
            if P["chain"][q]:
                rows.add(int(P["brow"][q]) * s + int(P["meta"][q]))
            else:
                for l in range(int(P["lanes"][q])):
                    rows.add(int(P["brow"][q]) * s + int(P["lane"][P["meta"][q] + l] >> 8))
        rows = np.array(sorted(rows), np.int64)
        assert rows.size > 0
        np.testing.assert_array_equal(y[rows], ref[rows], err_msg=coo.name)
        others = np.setdiff1d(np.arange(coo.m), rows)
        np.testing.assert_array_equal(y[others], y0[others])  # untouched


@pytest.mark.parametrize("s", [16, 64])
def test_oracle_slices_layout_rules(s):
    for coo in cases():
        b = oracle.build(coo.rows, coo.cols, coo.vals, coo.m, coo.n, s)
        P = b.slices(1e9)
        if P["slices"] == 0:
            continue
        M = (coo.m + s - 1) // s
        seg = segments(M)
        vidx = P["vidx"]
        used = vidx[vidx >= 0]
        assert np.unique(used).size == used.size == P["elements"], coo.name  # each element at one slot
        last_len = {}
        for q in range(P["slices"]):
            base, steps, lanes = int(P["base"][q]), int(P["steps"][q]), int(P["lanes"][q])
            if P["chain"][q]:
                assert steps > 256 and lanes == 1
                cols = P["words"][base:base + steps].astype(np.int64)
                assert np.all(np.diff(cols) > 0)
                continue
            brow = int(P["brow"][q])
            assert brow in seg[:-1], (coo.name, brow)  # a segment's first block row
            g = seg.index(brow)
            lens = []
            for l in range(lanes):
                rec = int(P["lane"][P["meta"][q] + l])
                off, n = rec >> 8, (rec & 255) + 1
                row = brow * s + off
                assert seg[g] * s <= row < seg[g + 1] * s  # inside the segment
                assert n <= 256
                lens.append(n)
                w = P["words"][base + l:base + 32 * n:32].astype(np.int64)
                cols = np.cumsum(w)  # deltas, the first absolute
                assert np.all(np.diff(cols) > 0) and cols[-1] < coo.n
                got = np.sort(coo.cols[coo.rows == row])
                np.testing.assert_array_equal(cols, got)
            assert lens == sorted(lens, reverse=True) and lens[0] == steps
            assert all(P["lane"][P["meta"][q] + l] == 0 for l in range(lanes, 32))
            # longest first within a segment, across its slices
            assert last_len.get(g, 1 << 30) >= lens[0]
            last_len[g] = lens[-1]
