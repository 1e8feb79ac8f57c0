"""Row-sharded SpMV over several GPUs, one process per GPU.

Each rank owns a contiguous range of block rows of A (balanced by
nonzeros) and the matching slice of y; x is split into equal slices, one per
rank, and all-gathered before every product -- the one exchange step of a
sharded SpMV.  The local product is the single-GPU kernel on the rank's rows,
so every y element is bitwise what one GPU computes: a row's sum never
crosses ranks.

The host logic (partition, element selection, the x exchange) runs with any
torch.distributed backend; the tests run it on two gloo ranks on the CPU.
"""
from __future__ import annotations

import numpy as np


def partition_block_rows(rows: np.ndarray, m: int, s: int, world: int) -> list[tuple[int, int]]:
    """Contiguous row ranges [r0, r1), one per rank, on block-row boundaries
    (multiples of s, the last ending at m), with about equal nonzeros each."""
    if world < 1 or s < 1 or m < 1:
        raise ValueError("world, s and m must be positive")
    M = -(-m // s)
    per_brow = np.bincount(np.asarray(rows, np.int64) // s, minlength=M)
    cum = np.concatenate([[0], np.cumsum(per_brow)])
    total = int(cum[-1])
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(cum, target, side="left"))
        cuts.append(min(max(b, cuts[-1]), M))
    cuts.append(M)
    return [(cuts[r] * s, min(cuts[r + 1] * s, m)) for r in range(world)]


def x_slices(n: int, world: int) -> list[tuple[int, int]]:
    """Equal slices of x (the last shorter), one per rank."""
    w = -(-n // world)
    return [(min(r * w, n), min((r + 1) * w, n)) for r in range(world)]


def local_elements(rows, cols, vals, r0: int, r1: int):
    """The elements of rows [r0, r1), rows renumbered from 0."""
    rows = np.asarray(rows, np.int64)
    keep = (rows >= r0) & (rows < r1)
    return rows[keep] - r0, np.asarray(cols, np.int64)[keep], None if vals is None else np.asarray(vals)[keep]


def gather_x(x_local, n: int, group=None):
    """The full x from every rank's slice (x_slices): one all-gather of equal,
    zero-padded slices."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    w = -(-n // world)
    buf = torch.zeros(w, dtype=x_local.dtype, device=x_local.device)
    buf[: x_local.numel()] = x_local
    out = torch.empty(world * w, dtype=x_local.dtype, device=x_local.device)
    dist.all_gather_into_tensor(out, buf, group=group)
    return out[:n]


class ShardedMatrix:
    """A's block rows [row0, row1) on this rank's GPU (an AbhsfMatrix of the
    rank's rows); spmv(x_local, y_local) gathers x and adds A_rank x onto the
    rank's slice of y."""

    def __init__(self, rows, cols, vals, m: int, n: int, block_size: int = 64, group=None, **build):
        import torch.distributed as dist

        from .matrix import AbhsfMatrix
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.m, self.n = int(m), int(n)
        self.ranges = partition_block_rows(rows, m, block_size, self.world)
        self.row0, self.row1 = self.ranges[self.rank]
        self.x0, self.x1 = x_slices(n, self.world)[self.rank]
        lr, lc, lv = local_elements(rows, cols, vals, self.row0, self.row1)
        self.local = None  # a rank without rows still takes part in the exchange
        if self.row1 > self.row0:
            self.local = AbhsfMatrix.from_elements(lr, lc, lv, self.row1 - self.row0, n, block_size=block_size,
                                                   **build)

    def spmv(self, x_local, y_local) -> None:
        """y_local += A[row0:row1, :] x, x given as this rank's slice
        x[x0:x1] (CUDA tensors).  Every rank calls it (the exchange is
        collective)."""
        x = gather_x(x_local, self.n, self.group)
        if self.local is not None:
            self.local.spmv(x, y_local)

    def release(self) -> None:
        if self.local is not None:
            self.local.release()
            self.local = None
