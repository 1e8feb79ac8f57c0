"""Row-sharded SpMV over several GPUs, one process per GPU.

Each rank owns a contiguous range of block rows of A (balanced by the
bytes their SpMV streams, or by nonzeros) and the matching slice of y; x is
split into equal slices, one per rank, and brought in before every product
-- the one exchange step of a sharded SpMV: all of it (an all-gather), or
only the entries the rank's columns read (a halo, HaloPlan).  The local product is the single-GPU kernel on the rank's rows,
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


def partition_block_rows(rows: np.ndarray, m: int, s: int, world: int, weights=None) -> list[tuple[int, int]]:
    """Contiguous row ranges [r0, r1), one per rank, on block-row boundaries
    (multiples of s, the last ending at m), with about equal weight each:
    `weights` per block row (block_row_bytes), else the nonzeros."""
    if world < 1 or s < 1 or m < 1:
        raise ValueError("world, s and m must be positive")
    M = -(-m // s)
    if weights is None:
        per_brow = np.bincount(np.asarray(rows, np.int64) // s, minlength=M)
    else:
        per_brow = np.asarray(weights, np.float64)
        if per_brow.shape != (M,) or np.any(per_brow < 0):
            raise ValueError("weights: one non-negative number per block row")
    cum = np.concatenate([[0], np.cumsum(per_brow)])
    total = float(cum[-1])
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(cum, target, side="left"))
        cuts.append(min(max(b, cuts[-1]), M))
    cuts.append(M)
    # a rank past the last block row gets the empty range (m, m)
    return [(min(cuts[r] * s, m), min(cuts[r + 1] * s, m)) for r in range(world)]


def block_row_bytes(rows, cols, m: int, n: int, s: int, value_bytes: int = 8) -> np.ndarray:
    """Bytes one SpMV streams for each block row, by the format's cost model:
    per occupied s x s tile the least-storage scheme's index bits
    (include/abhsf/msmf.h:35-63) plus 2 tag bits, plus its values, plus a
    block-column index and a tile header (8 bytes), plus the s entries of x
    it reads.  The weight for balancing ranks by bytes rather than by
    nonzeros: a bitmap or dense tile streams more per nonzero than a COO one."""
    from .matrix import block_scheme_bits, block_select_scheme
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    M, N = -(-m // s), -(-n // s)
    key = (rows // s) * N + cols // s
    tiles, z = np.unique(key, return_counts=True)
    zs, inv = np.unique(z, return_inverse=True)
    bits = np.array([block_scheme_bits(block_select_scheme(s, s, int(q), 8 * value_bytes), s, s, int(q),
                                       8 * value_bytes) for q in zs], np.float64)
    tile_bytes = (bits[inv] + 2) / 8 + value_bytes * z + 8 + 8 * s
    return np.bincount(tiles // N, weights=tile_bytes, minlength=M)


def x_slices(n: int, world: int) -> list[tuple[int, int]]:
    """Equal slices of x (the last shorter), one per rank."""
    w = -(-n // world)
    return [(min(r * w, n), min((r + 1) * w, n)) for r in range(world)]


def local_elements(rows, cols, vals, r0: int, r1: int):
    """The elements of rows [r0, r1), rows renumbered from 0."""
    rows = np.asarray(rows, np.int64)
    keep = (rows >= r0) & (rows < r1)
    return rows[keep] - r0, np.asarray(cols, np.int64)[keep], None if vals is None else np.asarray(vals)[keep]


def owners_of(idx: np.ndarray, owners: list[tuple[int, int]]) -> np.ndarray:
    """The rank whose range [r0, r1) holds each index (ranges contiguous,
    in rank order, possibly empty)."""
    ends = np.array([r1 for _, r1 in owners], np.int64)
    return np.searchsorted(ends, np.asarray(idx, np.int64), side="right")


class HaloPlan:
    """The entries of a distributed vector that this rank's elements read,
    fetched from the ranks that hold them: one all_to_all per product with
    exactly those entries, instead of an all-gather of the whole vector.

    `need` are the distinct columns of this rank's elements, ascending; the
    rank's local matrix is built on columns renumbered to positions in
    `need` (local_columns), a map that keeps column order, so every row's
    sum runs in the same order and gives the same bits as on the whole x.
    `owners` are the ranges of the vector each rank holds.  Built
    collectively (every rank, once): the index lists go to their owners in
    one all_to_all."""

    def __init__(self, cols, owners: list[tuple[int, int]], group=None, device=None):
        import torch
        import torch.distributed as dist
        world = dist.get_world_size(group)
        if len(owners) != world:
            raise ValueError("one owner range per rank")
        self.group = group
        self.need = np.unique(np.asarray(cols, np.int64))
        if self.need.size and (self.need[0] < 0 or self.need[-1] >= owners[-1][1]):
            raise ValueError("a column lies outside the owners' ranges")
        own = owners_of(self.need, owners)
        self.recv_counts = np.bincount(own, minlength=world).astype(np.int64)
        dev = torch.device("cpu") if device is None else torch.device(device)
        want = torch.from_numpy(self.recv_counts.copy()).to(dev)
        give = torch.empty(world, dtype=torch.int64, device=dev)
        dist.all_to_all_single(give, want, group=group)
        self.send_counts = give.cpu().numpy()
        # each owner receives the positions (in its own slice) the requesters read
        offsets = self.need - np.array([r0 for r0, _ in owners], np.int64)[own]
        idx = torch.empty(int(self.send_counts.sum()), dtype=torch.int64, device=dev)
        dist.all_to_all_single(idx, torch.from_numpy(offsets).to(dev), self.send_counts.tolist(),
                               self.recv_counts.tolist(), group=group)
        self.send_idx = idx
        self.device = dev

    @property
    def width(self) -> int:
        """Columns of the rank's local matrix (at least 1)."""
        return max(int(self.need.size), 1)

    def local_columns(self, cols) -> np.ndarray:
        return np.searchsorted(self.need, np.asarray(cols, np.int64))

    def halo_entries(self, rank: int) -> int:
        """Entries this rank receives from other ranks per product."""
        return int(self.recv_counts.sum() - self.recv_counts[rank])

    def fetch(self, v_local):
        """The needed entries (length `width`, in `need` order) from every
        rank's slice; v_local is this rank's slice.  Every rank calls it."""
        import torch
        import torch.distributed as dist
        out = torch.zeros(self.width, dtype=v_local.dtype, device=v_local.device)
        send = v_local[self.send_idx] if self.send_idx.numel() else v_local.new_empty(0)
        dist.all_to_all_single(out[: self.need.size], send.contiguous(), self.recv_counts.tolist(),
                               self.send_counts.tolist(), group=self.group)
        return out


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
       max_iters: int = 100000, group=None, fetch=None) -> dict:
    """FP64 conjugate gradients on a square SPD A whose rows, and the
    entries of b and x, are split over the ranks by `ranges` (the same
    ranges for rows and vector entries).

    local_spmv(v, q) adds this rank's rows of A times v onto q (its length
    r1 - r0), v being the full vector, or with `fetch` (a HaloPlan's, owners
    = ranges) the entries fetch(v_local) returns.  Each iteration is one
    exchange of the search direction and two all-reduced scalars (p.Ap and
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
        local_spmv(gather_ranges(v, ranges, group) if fetch is None else fetch(v), q)
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
    rank's rows); spmv(x_local, y_local) brings in x and adds A_rank x onto
    the rank's slice of y.

    balance: "bytes" splits the block rows by the bytes their SpMV streams
    (block_row_bytes), "nnz" by nonzeros.  exchange: "allgather" brings in
    all of x before each product; "halo" only the entries the rank's
    columns read (HaloPlan: for banded and stencil matrices a few planes of
    x instead of all of it), with the local matrix on renumbered columns.
    Either way y is bitwise the one-GPU result (with sum_order
    "reference", the default)."""

    def __init__(self, rows, cols, vals, m: int, n: int, block_size: int = 64, group=None,
                 exchange: str = "allgather", balance: str = "bytes", **build):
        import torch
        import torch.distributed as dist

        from .matrix import AbhsfMatrix
        if exchange not in ("allgather", "halo"):
            raise ValueError("exchange: allgather or halo")
        if balance not in ("bytes", "nnz"):
            raise ValueError("balance: bytes or nnz")
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.m, self.n = int(m), int(n)
        self.exchange = exchange
        weights = None
        if balance == "bytes" and self.world > 1:
            vb = {"f64": 8, "f32": 4, "bf16": 2}.get(build.get("value_type", "f64"), 8)
            weights = block_row_bytes(rows, cols, m, n, block_size, vb)
        self.ranges = partition_block_rows(rows, m, block_size, self.world, weights)
        self.row0, self.row1 = self.ranges[self.rank]
        self.x0, self.x1 = x_slices(n, self.world)[self.rank]
        lr, lc, lv = local_elements(rows, cols, vals, self.row0, self.row1)
        self._cols = lc
        self.halo = self._halo_cg = None
        width = n
        if exchange == "halo":
            dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else None
            self._device = dev
            self.halo = HaloPlan(lc, x_slices(n, self.world), group, dev)
            lc = self.halo.local_columns(lc)
            width = self.halo.width
        self.local = None  # a rank without rows still takes part in the exchange
        if self.row1 > self.row0:
            self.local = AbhsfMatrix.from_elements(lr, lc, lv, self.row1 - self.row0, width, block_size=block_size,
                                                   **build)

    def _x(self, x_local):
        if self.halo is not None:
            return self.halo.fetch(x_local)
        return gather_x(x_local, self.n, self.group)

    def spmv(self, x_local, y_local) -> None:
        """y_local += A[row0:row1, :] x, x given as this rank's slice
        x[x0:x1] (CUDA tensors).  Every rank calls it (the exchange is
        collective)."""
        x = self._x(x_local)
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
        fetch = None
        if self.exchange == "halo":
            # the CG vectors live on the row ranges, not on the x slices
            if self._halo_cg is None:
                self._halo_cg = HaloPlan(self._cols, self.ranges, self.group, self._device)
            fetch = self._halo_cg.fetch

        def local_spmv(v, q):
            if self.local is not None:
                self.local.spmv(v, q)
        return cg(local_spmv, b_local, x_local, self.ranges, rtol, max_iters, self.group, fetch)

    def release(self) -> None:
        if self.local is not None:
            self.local.release()
            self.local = None
