"""Row-sharded SpMV host logic on two CPU ranks (gloo): the block-row
partition, each rank's elements, and the x all-gather compose to the full
product.  The local products here are the oracle's (the checker); on GPUs
they are the library's kernel on each rank's rows."""
import os
import socket

import numpy as np
import pytest

from abhsf_b200 import sharded
from abhsf_b200 import workloads as W


def test_partition_covers_rows_on_block_boundaries():
    coo = W.rmat(5000, 8, seed=3)
    for world in (1, 2, 3, 8):
        for s in (32, 64):
            parts = sharded.partition_block_rows(coo.rows, coo.m, s, world)
            assert len(parts) == world and parts[0][0] == 0 and parts[-1][1] == coo.m
            for (a0, a1), (b0, b1) in zip(parts, parts[1:]):
                assert a1 == b0 and a0 <= a1 and a0 % s == 0
            counts = [int(((coo.rows >= a) & (coo.rows < b)).sum()) for a, b in parts]
            assert sum(counts) == coo.nnz
            if world <= 2:  # balanced to within one block row's nonzeros
                per_brow = np.bincount(coo.rows // s).max()
                assert max(counts) - coo.nnz / world <= per_brow
    assert sharded.x_slices(10, 3) == [(0, 4), (4, 8), (8, 10)]
    with pytest.raises(ValueError):
        sharded.partition_block_rows(coo.rows, coo.m, 64, 0)


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    from oracle import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        coo = W.random_blocky(1000, 900, 64, 80, seed=7)
        x = W.rhs(coo.n, 1)
        y0 = W.rhs(coo.m, 2)
        r0, r1 = sharded.partition_block_rows(coo.rows, coo.m, 64, world)[rank]
        x0, x1 = sharded.x_slices(coo.n, world)[rank]
        xfull = sharded.gather_x(torch.from_numpy(x[x0:x1].copy()), coo.n).numpy()
        lr, lc, lv = sharded.local_elements(coo.rows, coo.cols, coo.vals, r0, r1)
        order = np.lexsort((lc, lr))
        y = oracle.spmv_elements(lr[order], lc[order], lv[order], xfull, y0[r0:r1].copy())
        out.put((rank, r0, r1, bool(np.array_equal(xfull, x)), y))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_compose_the_full_product():
    import torch.multiprocessing as mp
    from oracle import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    coo = W.random_blocky(1000, 900, 64, 80, seed=7)
    x = W.rhs(coo.n, 1)
    y0 = W.rhs(coo.m, 2)
    order = np.lexsort((coo.cols, coo.rows))
    want = oracle.spmv_elements(coo.rows[order], coo.cols[order], coo.vals[order], x, y0.copy())
    assert all(r[3] for r in res)  # every rank gathered the whole x
    y = np.concatenate([r[4] for r in res])
    assert res[0][1] == 0 and res[0][2] == res[1][1] and res[1][2] == coo.m
    np.testing.assert_array_equal(y, want)  # row sums never cross ranks: bitwise the one-GPU order


def test_partition_gives_empty_ranges_past_the_last_block_row():
    assert sharded.partition_block_rows(np.arange(50), 50, 64, 2) == [(0, 50), (50, 50)]
    parts = sharded.partition_block_rows(np.arange(200) % 130, 130, 64, 4)
    assert parts[0][0] == 0 and parts[-1][1] == 130
    for a0, a1 in parts:
        assert 0 <= a0 <= a1 <= 130
    for (a0, a1), (b0, b1) in zip(parts, parts[1:]):
        assert a1 == b0


def _cg_ref(coo, b, rtol, max_iters):
    """One-process CG with the sharded solver's recurrences (numpy, f64)."""
    from oracle import oracle

    def A(v):
        return oracle.spmv_elements(coo.rows, coo.cols, coo.vals, v, np.zeros(coo.m))
    x = np.zeros(coo.n)
    bb = float(b @ b)
    r = b - A(x)
    p = r.copy()
    rr = float(r @ r)
    it = 0
    while rr > rtol * rtol * bb and it < max_iters:
        q = A(p)
        alpha = rr / float(p @ q)
        x += alpha * p
        r -= alpha * q
        rr_new = float(r @ r)
        p = r + (rr_new / rr) * p
        rr = rr_new
        it += 1
    return x, it


def _cg_rank_main(rank, world, port, g, out):
    import datetime

    import torch
    import torch.distributed as dist
    from oracle import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        coo = W.laplacian_2d(g)
        b = W.rhs(coo.n, 5)
        ranges = sharded.partition_block_rows(coo.rows, coo.m, 64, world)
        r0, r1 = ranges[rank]
        lr, lc, lv = sharded.local_elements(coo.rows, coo.cols, coo.vals, r0, r1)

        def local_spmv(v, q):  # the oracle's product on this rank's rows (the checker)
            q.copy_(torch.from_numpy(oracle.spmv_elements(lr, lc, lv, v.numpy(), q.numpy().copy())))
        xl = torch.zeros(r1 - r0, dtype=torch.float64)
        info = sharded.cg(local_spmv, torch.from_numpy(b[r0:r1].copy()), xl, ranges, rtol=1e-10, max_iters=2000)
        full = sharded.gather_ranges(xl, ranges).numpy()
        out.put((rank, r0, r1, info, xl.numpy().copy(), full))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,g", [(3, 24), (2, 7)])
def test_gloo_ranks_sharded_cg_converges_like_one_process(world, g):
    """Rows, b and x split by block rows over the ranks (g = 7: 49 rows, one
    block row, so rank 1 owns nothing and still takes part in every
    exchange); the solution, residual and iteration count agree with a
    one-process CG of the same recurrences."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_cg_rank_main, args=(r, world, port, g, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    coo = W.laplacian_2d(g)
    b = W.rhs(coo.n, 5)
    x_ref, it_ref = _cg_ref(coo, b, 1e-10, 2000)
    x = np.concatenate([r[4] for r in res])
    assert x.size == coo.n
    for r in res:
        np.testing.assert_array_equal(r[5], x)  # every rank gathered the same full vector
        assert r[3]["converged"] and r[3]["rel_residual"] <= 1e-10
        assert r[3]["iterations"] == res[0][3]["iterations"]
    assert abs(res[0][3]["iterations"] - it_ref) <= 2
    dense = np.zeros((coo.n, coo.n))
    dense[coo.rows, coo.cols] = coo.vals
    exact = np.linalg.solve(dense, b)
    assert np.linalg.norm(x - exact) <= 1e-7 * np.linalg.norm(exact)
    assert np.linalg.norm(x - x_ref) <= 1e-7 * np.linalg.norm(x_ref)
    if g == 7:
        assert res[1][1] == res[1][2] == coo.m  # the empty rank


def test_block_row_bytes_weigh_the_format():
    """Per block row: the least-storage scheme's bits, the values, a tile
    header and an x block per tile; a row of bitmap tiles weighs more per
    nonzero than a row of COO tiles, and the weights balance the ranks."""
    from abhsf_b200 import matrix as mx
    s = 64
    # block row 0: one tile with 2000 nonzeros (bitmap); block row 1: 100 tiles of 20 (COO)
    r0 = np.repeat(np.arange(64), 32)[:2000]
    c0 = np.tile(np.arange(0, 64, 2), 64)[:2000]
    r1 = 64 + np.tile(np.arange(20), 100)
    c1 = np.repeat(np.arange(100) * 64, 20) + np.tile(np.arange(20), 100)
    rows, cols = np.concatenate([r0, r1]), np.concatenate([c0, c1])
    w = sharded.block_row_bytes(rows, cols, 128, 6400, s)
    assert mx.block_select_scheme(s, s, 2000) == "bitmap" and mx.block_select_scheme(s, s, 20) == "coo"
    want0 = (mx.block_scheme_bits("bitmap", s, s, 2000) + 2) / 8 + 8 * 2000 + 8 + 8 * s
    want1 = 100 * ((mx.block_scheme_bits("coo", s, s, 20) + 2) / 8 + 8 * 20 + 8 + 8 * s)
    np.testing.assert_allclose(w, [want0, want1])
    assert w[0] / 2000 < w[1] / 2000  # same nonzeros; many COO tiles read many x blocks
    coo = W.tiled_mixture(n=8192, tile=64, p=0.02, seed=4)
    wb = sharded.block_row_bytes(coo.rows, coo.cols, coo.m, coo.n, 64)
    parts = sharded.partition_block_rows(coo.rows, coo.m, 64, 4, weights=wb)
    got = [wb[a // 64: -(-b // 64)].sum() for a, b in parts]
    assert abs(sum(got) - wb.sum()) < 1e-6 * wb.sum()
    assert max(got) - wb.sum() / 4 <= wb.max()
    with pytest.raises(ValueError):
        sharded.partition_block_rows(coo.rows, coo.m, 64, 4, weights=wb[:-1])


def _halo_rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    from oracle import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = {}
        # SpMV: a banded matrix, x held in equal slices
        coo = W.banded(3000, 40, seed=2)
        x = W.rhs(coo.n, 1)
        y0 = W.rhs(coo.m, 2)
        wb = sharded.block_row_bytes(coo.rows, coo.cols, coo.m, coo.n, 64)
        r0, r1 = sharded.partition_block_rows(coo.rows, coo.m, 64, world, wb)[rank]
        x0, x1 = sharded.x_slices(coo.n, world)[rank]
        lr, lc, lv = sharded.local_elements(coo.rows, coo.cols, coo.vals, r0, r1)
        plan = sharded.HaloPlan(lc, sharded.x_slices(coo.n, world))
        xc = plan.fetch(torch.from_numpy(x[x0:x1].copy())).numpy()
        res["fetched_ok"] = bool(np.array_equal(xc[: plan.need.size], x[plan.need]))
        res["halo"] = plan.halo_entries(rank)
        order = np.lexsort((lc, lr))
        res["y"] = oracle.spmv_elements(lr[order], plan.local_columns(lc[order]), lv[order], xc,
                                        y0[r0:r1].copy())
        res["r"] = (r0, r1)
        # CG on the 2D Laplacian: halo exchange against all-gather
        lap = W.laplacian_2d(20)
        b = W.rhs(lap.n, 5)
        ranges = sharded.partition_block_rows(lap.rows, lap.m, 64, world)
        q0, q1 = ranges[rank]
        lr, lc, lv = sharded.local_elements(lap.rows, lap.cols, lap.vals, q0, q1)
        hp = sharded.HaloPlan(lc, ranges)
        lcc = hp.local_columns(lc)

        def full_product(v, q):
            q.copy_(torch.from_numpy(oracle.spmv_elements(lr, lc, lv, v.numpy(), q.numpy().copy())))

        def halo_product(v, q):
            q.copy_(torch.from_numpy(oracle.spmv_elements(lr, lcc, lv, v.numpy(), q.numpy().copy())))
        xa = torch.zeros(q1 - q0, dtype=torch.float64)
        xh = torch.zeros(q1 - q0, dtype=torch.float64)
        bl = torch.from_numpy(b[q0:q1].copy())
        res["cg_all"] = sharded.cg(full_product, bl, xa, ranges, 1e-10, 2000)
        res["cg_halo"] = sharded.cg(halo_product, bl, xh, ranges, 1e-10, 2000, fetch=hp.fetch)
        res["cg_same_bits"] = bool(np.array_equal(xa.numpy().view(np.uint64), xh.numpy().view(np.uint64)))
        res["cg_halo_entries"] = hp.halo_entries(rank)
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_halo_exchange_gives_the_full_product_bits(world):
    """Each rank fetches only the x entries its columns read (a banded
    matrix: its slice and about a band's width from each neighbour); the
    products on renumbered columns compose to the full product bit for bit,
    and CG through the halo exchange retraces CG through the all-gather
    bit for bit."""
    import torch.multiprocessing as mp
    from oracle import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_halo_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [r for _, r in sorted((q.get(timeout=180) for _ in procs), key=lambda t: t[0])]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    coo = W.banded(3000, 40, seed=2)
    x = W.rhs(coo.n, 1)
    y0 = W.rhs(coo.m, 2)
    order = np.lexsort((coo.cols, coo.rows))
    want = oracle.spmv_elements(coo.rows[order], coo.cols[order], coo.vals[order], x, y0.copy())
    assert all(r["fetched_ok"] for r in res)
    assert res[0]["r"][0] == 0 and res[-1]["r"][1] == coo.m
    np.testing.assert_array_equal(np.concatenate([r["y"] for r in res]), want)
    # a rank reads columns [r0 - 40, r1 + 40) and holds x[x0:x1): it fetches at
    # most the difference (none when its rows sit inside its slice)
    for r, (x0, x1) in zip(res, sharded.x_slices(coo.n, world)):
        r0, r1 = r["r"]
        assert 0 <= r["halo"] <= abs(r0 - x0) + abs(r1 - x1) + 2 * 40
    assert sum(r["halo"] for r in res) > 0
    for r in res:
        assert r["cg_all"]["converged"] and r["cg_same_bits"]
        assert r["cg_halo"] == r["cg_all"]
        assert 0 < r["cg_halo_entries"] <= 2 * 20  # one grid row from each neighbour


def _halo_empty_rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    from oracle import oracle
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        coo = W.laplacian_2d(7)  # 49 rows, one block row: rank 1 owns no rows
        x = W.rhs(coo.n, 1)
        r0, r1 = sharded.partition_block_rows(coo.rows, coo.m, 64, world)[rank]
        x0, x1 = sharded.x_slices(coo.n, world)[rank]
        lr, lc, lv = sharded.local_elements(coo.rows, coo.cols, coo.vals, r0, r1)
        plan = sharded.HaloPlan(lc, sharded.x_slices(coo.n, world))
        xc = plan.fetch(torch.from_numpy(x[x0:x1].copy())).numpy()
        y = oracle.spmv_elements(lr, plan.local_columns(lc), lv, xc, np.zeros(r1 - r0))
        out.put((rank, (r0, r1), int(plan.need.size), int(plan.send_counts.sum()), plan.width, y))
    finally:
        dist.destroy_process_group()


def test_gloo_halo_with_a_rank_that_reads_nothing():
    """A rank without rows needs no x entries (its fetch is a zero-length
    receive, its local width 1) but still sends the part of x it holds."""
    import torch.multiprocessing as mp
    from oracle import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_halo_empty_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    coo = W.laplacian_2d(7)
    assert res[0][1] == (0, 49) and res[1][1] == (49, 49)
    assert res[0][2] == 49 and res[1][2] == 0 and res[1][4] == 1
    assert res[0][3] == 25 and res[1][3] == 24  # each sends what rank 0 reads of its slice
    want = oracle.spmv_elements(coo.rows, coo.cols, coo.vals, W.rhs(coo.n, 1), np.zeros(coo.m))
    np.testing.assert_array_equal(res[0][5], want)
    assert res[1][5].size == 0


class _OracleLocal:
    """Stands in for the rank's GPU matrix in ShardedMatrix on gloo ranks: the
    oracle's product (the checker) on the same elements."""

    def __init__(self, rows, cols, vals, m, n):
        order = np.lexsort((cols, rows))
        self.rows, self.cols, self.vals = rows[order], cols[order], np.asarray(vals)[order]
        self.m, self.n = m, n

    @classmethod
    def from_elements(cls, rows, cols, vals, m, n, block_size=64, **build):
        return cls(np.asarray(rows), np.asarray(cols), vals, m, n)

    def spmv(self, x, y):
        import torch
        from oracle import oracle
        assert x.numel() == self.n and y.numel() == self.m
        y.copy_(torch.from_numpy(oracle.spmv_elements(self.rows, self.cols, self.vals, x.numpy(), y.numpy().copy())))

    def release(self):
        pass


def _class_rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    from abhsf_b200 import matrix as mxm
    mxm.AbhsfMatrix = _OracleLocal
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        res = {}
        coo = W.banded(2000, 30, seed=4)
        x = W.rhs(coo.n, 1)
        y0 = W.rhs(coo.m, 2)
        for ex in ("allgather", "halo"):
            S = sharded.ShardedMatrix(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64, exchange=ex)
            y = torch.from_numpy(y0[S.row0:S.row1].copy())
            S.spmv(torch.from_numpy(x[S.x0:S.x1].copy()), y)
            res["spmv_" + ex] = (S.row0, S.row1, y.numpy().copy())
            if ex == "halo":
                res["halo_width"] = S.local.n if S.local is not None else 0
            S.release()
        lap = W.laplacian_2d(20)
        b = W.rhs(lap.n, 5)
        for ex in ("allgather", "halo"):
            S = sharded.ShardedMatrix(lap.rows, lap.cols, lap.vals, lap.m, lap.n, block_size=64, exchange=ex)
            xs = torch.zeros(S.row1 - S.row0, dtype=torch.float64)
            info = S.cg(torch.from_numpy(b[S.row0:S.row1].copy()), xs, rtol=1e-10, max_iters=2000)
            res["cg_" + ex] = (info, xs.numpy().copy())
            S.release()
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_gloo_sharded_matrix_class_both_exchanges():
    """ShardedMatrix on three gloo ranks, its local GPU matrix replaced by
    the oracle's product: y composes to the full product bit for bit with
    either exchange (the halo rank's matrix is only as wide as the columns it
    reads), and CG gives the same bits and iterations with either."""
    import torch.multiprocessing as mp
    from oracle import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 3
    procs = [ctx.Process(target=_class_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [r for _, r in sorted((q.get(timeout=180) for _ in procs), key=lambda t: t[0])]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    coo = W.banded(2000, 30, seed=4)
    x = W.rhs(coo.n, 1)
    y0 = W.rhs(coo.m, 2)
    order = np.lexsort((coo.cols, coo.rows))
    want = oracle.spmv_elements(coo.rows[order], coo.cols[order], coo.vals[order], x, y0.copy())
    for ex in ("allgather", "halo"):
        parts = [r["spmv_" + ex] for r in res]
        assert parts[0][0] == 0 and parts[-1][1] == coo.m
        np.testing.assert_array_equal(np.concatenate([p[2] for p in parts]), want)
    for r in res:
        r0, r1 = r["spmv_halo"][:2]
        assert 0 < r["halo_width"] <= (r1 - r0) + 2 * 30  # its rows' band, not all 2000 columns
        a_info, a_x = r["cg_allgather"]
        h_info, h_x = r["cg_halo"]
        assert a_info["converged"] and a_info == h_info
        np.testing.assert_array_equal(a_x.view(np.uint64), h_x.view(np.uint64))


def test_partition_properties_on_generated_inputs():
    hyp = pytest.importorskip("hypothesis")
    st = pytest.importorskip("hypothesis.strategies")

    @hyp.settings(max_examples=300, deadline=None, derandomize=True)
    @hyp.given(m=st.integers(1, 5000), s=st.sampled_from([16, 32, 64, 128, 256]), world=st.integers(1, 9),
               k=st.integers(0, 3000), seed=st.integers(0, 10 ** 6), use_weights=st.booleans())
    def check(m, s, world, k, seed, use_weights):
        rng = np.random.default_rng(seed)
        rows = rng.integers(0, m, k)
        M = -(-m // s)
        w = rng.uniform(0, 5, M) if use_weights else None
        parts = sharded.partition_block_rows(rows, m, s, world, w)
        assert len(parts) == world and parts[0][0] == 0 and parts[-1][1] == m
        per = w if use_weights else np.bincount(rows // s, minlength=M).astype(float)
        got = []
        for r, (a, b) in enumerate(parts):
            assert 0 <= a <= b <= m and (a % s == 0 or a == m)
            if r + 1 < world:
                assert b == parts[r + 1][0]
            got.append(per[a // s: -(-b // s)].sum() if b > a else 0.0)
        assert abs(sum(got) - per.sum()) <= 1e-9 * max(per.sum(), 1.0)
        # each cut lands at the first block row where the prefix reaches its target
        assert max(got) <= per.sum() / world + (per.max() if per.size else 0.0) + 1e-9

    check()
