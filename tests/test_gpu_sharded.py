"""The row-sharded SpMV on one GPU (a one-rank NCCL group): the gather and
the local kernel give abhsf_spmv's y bit for bit.  More ranks need more GPUs
than a run here has; their host logic is tested on gloo ranks."""
import socket

import numpy as np
import pytest

from abhsf_b200 import AbhsfMatrix
from abhsf_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_one_rank_sharded_spmv_equals_spmv(gpu):
    import datetime

    import torch
    import torch.distributed as dist
    from abhsf_b200.sharded import ShardedMatrix
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        coo = W.random_blocky(3000, 2500, 64, 200, seed=9)
        x = torch.from_numpy(W.rhs(coo.n, 1)).cuda()
        y0 = torch.from_numpy(W.rhs(coo.m, 2)).cuda()
        A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
        want = y0.clone()
        A.spmv(x, want)
        S = ShardedMatrix(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
        assert (S.row0, S.row1, S.x0, S.x1) == (0, coo.m, 0, coo.n)
        y = y0.clone()
        S.spmv(x[S.x0:S.x1].contiguous(), y)
        torch.cuda.synchronize()
        assert torch.equal(y, want)
        S.release()
        A.release()
    finally:
        dist.destroy_process_group()


def test_one_rank_sharded_cg_matches_cg(gpu):
    """The sharded CG on a one-rank NCCL group (the library's SpMV on the
    rank's rows, the scalars all-reduced) solves the 2D Laplacian like
    abhsf_cg: both converge to rtol, to the same solution."""
    import datetime

    import torch
    import torch.distributed as dist
    from abhsf_b200 import cg
    from abhsf_b200.sharded import ShardedMatrix
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        coo = W.laplacian_2d(64)
        b = torch.from_numpy(W.rhs(coo.n, 5)).cuda()
        A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
        x1 = torch.zeros_like(b)
        want = cg(A, b, x1, rtol=1e-10, max_iters=5000)
        S = ShardedMatrix(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
        x2 = torch.zeros_like(b)
        got = S.cg(b[S.row0:S.row1], x2, rtol=1e-10, max_iters=5000)
        torch.cuda.synchronize()
        assert want["converged"] and got["converged"] and got["rel_residual"] <= 1e-10
        # the dot products round differently (one all-reduced torch.dot against the
        # library's block partials), so the trajectories part slightly
        assert abs(got["iterations"] - want["iterations"]) <= max(3, want["iterations"] // 50)
        # both lie within kappa * rtol (kappa ~ 1.7e3 at g = 64) of the exact solution
        assert torch.linalg.norm(x2 - x1) <= 1e-6 * torch.linalg.norm(x1)
        S.release()
        A.release()
    finally:
        dist.destroy_process_group()


def test_one_rank_halo_exchange_equals_spmv_and_cg(gpu):
    """The halo exchange on a one-rank NCCL group (the all_to_all of the
    needed x entries, the rank's matrix on renumbered columns): y is
    abhsf_spmv's bit for bit, and CG converges as through the all-gather."""
    import datetime

    import torch
    import torch.distributed as dist
    from abhsf_b200.sharded import ShardedMatrix
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        coo = W.random_blocky(3000, 2500, 64, 200, seed=9)
        x = torch.from_numpy(W.rhs(coo.n, 1)).cuda()
        y0 = torch.from_numpy(W.rhs(coo.m, 2)).cuda()
        A = AbhsfMatrix.from_elements(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64)
        want = y0.clone()
        A.spmv(x, want)
        S = ShardedMatrix(coo.rows, coo.cols, coo.vals, coo.m, coo.n, block_size=64, exchange="halo")
        assert S.halo.halo_entries(0) == 0 and S.local.n == np.unique(coo.cols).size
        y = y0.clone()
        S.spmv(x[S.x0:S.x1].contiguous(), y)
        torch.cuda.synchronize()
        assert torch.equal(y, want)
        S.release()
        A.release()
        lap = W.laplacian_2d(32)
        b = torch.from_numpy(W.rhs(lap.n, 5)).cuda()
        infos, xs = [], []
        for ex in ("allgather", "halo"):
            S = ShardedMatrix(lap.rows, lap.cols, lap.vals, lap.m, lap.n, block_size=64, exchange=ex)
            xv = torch.zeros_like(b)
            infos.append(S.cg(b, xv, rtol=1e-10, max_iters=3000))
            xs.append(xv)
            S.release()
        torch.cuda.synchronize()
        assert infos[0]["converged"] and infos[0] == infos[1]
        assert torch.equal(xs[0], xs[1])  # the same products in the same order
    finally:
        dist.destroy_process_group()
