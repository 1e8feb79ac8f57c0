"""The replica path's host logic on two CPU ranks (gloo): every rank times its
own steps, the job takes the slowest rank's time and counts every rank's
bytes.  No GPU: this is the logic bench.py runs under torchrun on N GPUs."""
import os
import socket

import pytest

from abhsf_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, lr, w = replicas.rank_info()
        slowest = replicas.max_over_ranks(times[rank])
        dist.barrier()
        out.put((r, lr, w, slowest, replicas.aggregate_rate(1e9, slowest, w)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    times = [0.004, 0.005]
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[:3] for r in res] == [(0, 0, 2), (1, 1, 2)]
    for r in res:
        assert r[3] == 0.005  # every rank sees the slowest rank's time
        assert r[4] == pytest.approx(2 * 1e9 / 0.005 / 1e9)  # both ranks' bytes over it


def test_single_process_without_group():
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.aggregate_rate(2e9, 0.5, 1) == pytest.approx(4.0)
    with pytest.raises(ValueError):
        replicas.aggregate_rate(1.0, 0.0, 1)
