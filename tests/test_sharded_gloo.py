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
