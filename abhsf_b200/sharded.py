"""Row-sharded SpMV over several GPUs, one process per GPU.

Each rank owns a contiguous range of block rows of A (balanced by
nonzeros) and the matching slice of y; x is split into equal slices, one per
rank, and all-gathered before every product -- the one exchange step of a
sharded SpMV.  The local product is the single-GPU kernel on the rank's rows,
so every y element is bitwise what one GPU computes: a row's sum never
crosses ranks.

CG over the shards (`cg`, `ShardedMatrix.cg`) splits b and x by the same
block-row ranges as the rows: per iteration one gather of the search
direction and two all-reduced scalars.

The host logic (partition, element selection, the exchanges, the CG
recurrences) runs with any torch.distributed backend; the tests run it on
gloo ranks on the CPU.
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
    # a rank past the last block row gets the empty range (m, m)
    return [(min(cuts[r] * s, m), min(cuts[r + 1] * s, m)) for r in range(world)]


def x_slices(n: int, world: int) -> list[tuple[int, int]]:
    """Equal slices of x (the last shorter), one per rank."""
    w = -(-n // world)
    return [(min(r * w, n), min((r + 1) * w, n)) for r in range(world)]


def local_elements(rows, cols, vals, r0: int, r1: int):
    """The elements of rows [r0, r1), rows renumbered from 0."""
    rows = np.asarray(rows, np.int64)
    keep = (rows >= r0) & (rows < r1)
    return rows[keep] - r0, np.asarray(cols, np.int64)[keep], None if vals is None else np.asarray(vals)[keep]


def gather_ranges(v_local, ranges: list[tuple[int, int]], group=None):
    """The full vector from every rank's slice v[r0:r1] (ranges of any
    lengths, one per rank, in order): one all-gather of slices zero-padded to
    the longest."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    if len(ranges) != world:
        raise ValueError("one range per rank")
    w = max(max(r1 - r0 for r0, r1 in ranges), 1)
    buf = torch.zeros(w, dtype=v_local.dtype, device=v_local.device)
    buf[: v_local.numel()] = v_local
    out = torch.empty(world * w, dtype=v_local.dtype, device=v_local.device)
    dist.all_gather_into_tensor(out, buf, group=group)
    return torch.cat([out[r * w: r * w + (r1 - r0)] for r, (r0, r1) in enumerate(ranges)])


def cg(local_spmv, b_local, x_local, ranges: list[tuple[int, int]], rtol: float = 1e-10,
       max_iters: int = 100000, group=None) -> dict:
    """FP64 conjugate gradients on a square SPD A whose rows, and the
    entries of b and x, are split over the ranks by `ranges` (the same
    ranges for rows and vector entries).

    local_spmv(v, q) adds this rank's rows of A times the full vector v onto
    q (its length r1 - r0).  Each iteration is one gather of the search
    direction (the SpMV's exchange) and two all-reduced scalars (p.Ap and
    r.r); the stopping rule and the returned fields are those of the
    one-GPU solver: |r| <= rtol |b|, with the final relative residual taken
    from a recomputed b - A x.  x_local (a tensor of this rank's entries) is
    the initial guess and receives the solution.  Every rank calls it."""
    import torch
    import torch.distributed as dist

    def dot(u, v):
        t = torch.dot(u, v).reshape(1) if u.numel() else torch.zeros(1, dtype=u.dtype, device=u.device)
        dist.all_reduce(t, group=group)
        return float(t.item())

    def matvec(v):
        q = torch.zeros_like(v)
        local_spmv(gather_ranges(v, ranges, group), q)
        return q

    bb = dot(b_local, b_local)
    tol2 = rtol * rtol * bb
    r = b_local - matvec(x_local)
    p = r.clone()
    rr = dot(r, r)
    iters = 0
    while rr > tol2 and iters < max_iters:
        q = matvec(p)
        pq = dot(p, q)
        alpha = rr / pq
        x_local.add_(p, alpha=alpha)
        r.add_(q, alpha=-alpha)
        rr_new = dot(r, r)
        p.mul_(rr_new / rr).add_(r)
        rr = rr_new
        iters += 1
    r = b_local - matvec(x_local)
    rr = dot(r, r)
    rel = (rr / bb) ** 0.5 if bb > 0 else rr ** 0.5
    return {"iterations": iters, "outer_iterations": 1, "converged": rel <= rtol, "rel_residual": rel}


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

    def cg(self, b_local, x_local, rtol: float = 1e-10, max_iters: int = 100000) -> dict:
        """Solves A x = b (A square, SPD) over all ranks; b_local and x_local
        are this rank's entries [row0, row1) (CUDA float64), x_local the
        initial guess, receiving the solution.  Every rank calls it."""
        if self.m != self.n:
            raise ValueError("CG needs a square matrix")
        for v in (b_local, x_local):
            if v.numel() != self.row1 - self.row0:
                raise ValueError("b_local and x_local hold this rank's rows [row0, row1)")

        def local_spmv(v, q):
            if self.local is not None:
                self.local.spmv(v, q)
        return cg(local_spmv, b_local, x_local, self.ranges, rtol, max_iters, self.group)

    def release(self) -> None:
        if self.local is not None:
            self.local.release()
            self.local = None
