"""Seeded synthetic sparse matrices with the shapes the ABHSF SpMV path is
measured on.  SuiteSparse matrices (block_statistics/experiments/matrices in
the reference) are not available offline; these generators stand in for them.

All generators return a :class:`Coo` with int64 row/column indices and float64
values, rows and columns 0-based (the convention of the reference's
matrix_market_reader, include/abhsf/utils/matrix_market_reader.h:135-136).
Randomness comes from numpy's PCG64 ``default_rng(seed)``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Coo:
    rows: np.ndarray  # int64 [nnz]
    cols: np.ndarray  # int64 [nnz]
    vals: np.ndarray  # float64 [nnz]
    m: int
    n: int
    name: str = ""

    @property
    def nnz(self) -> int:
        return int(self.rows.size)


def laplacian_2d(g: int = 512, diag: float = 4.0, off: float = -1.0) -> Coo:
    """5-point Laplacian on a g x g grid, i = gy*g + gx, elements in row-major
    order.  g = 512 gives n = 262,144 and nnz = 1,308,672."""
    n = g * g
    i = np.arange(n, dtype=np.int64)
    gx, gy = i % g, i // g
    parts = []
    # column order within a row: i-g, i-1, i, i+1, i+g
    for dc, mask, v in ((-g, gy > 0, off), (-1, gx > 0, off), (0, None, diag),
                        (1, gx < g - 1, off), (g, gy < g - 1, off)):
        r = i if mask is None else i[mask]
        parts.append((r, r + dc, np.full(r.size, v)))
    rows = np.concatenate([p[0] for p in parts])
    cols = np.concatenate([p[1] for p in parts])
    vals = np.concatenate([p[2] for p in parts])
    order = np.lexsort((cols, rows))
    return Coo(rows[order], cols[order], vals[order].astype(np.float64), n, n, f"laplace2d_{g}")


def laplacian_3d(g: int = 256, diag: float = 6.0, off: float = -1.0) -> Coo:
    """7-point Laplacian on a g^3 grid (SPD), elements in row-major order.
    g = 256 gives n = 16,777,216 and nnz = 117,047,296."""
    n = g ** 3
    i = np.arange(n, dtype=np.int64)
    gx, gy, gz = i % g, (i // g) % g, i // (g * g)
    parts = []
    for dc, mask, v in ((-g * g, gz > 0, off), (-g, gy > 0, off), (-1, gx > 0, off),
                        (0, None, diag), (1, gx < g - 1, off), (g, gy < g - 1, off),
                        (g * g, gz < g - 1, off)):
        r = i if mask is None else i[mask]
        parts.append((r, r + dc, v))
    rows = np.concatenate([p[0] for p in parts])
    cols = np.concatenate([p[1] for p in parts])
    vals = np.concatenate([np.full(p[0].size, p[2], dtype=np.float64) for p in parts])
    order = np.lexsort((cols, rows))
    return Coo(rows[order], cols[order], vals[order], n, n, f"laplace3d_{g}")


# Tile-occupancy probability that gives ~60M nnz for the tiled mixture below
# (52.7k occupied 64x64 tiles of 4.29e9).  The nominal p = 0.002 would give
# ~8.6M tiles and ~9.8e9 nnz, which contradicts the stated ~60M nnz.
TILED_MIXTURE_P = 1.2266e-5


def tiled_mixture(n: int = 4_194_304, tile: int = 64, p: float = TILED_MIXTURE_P, seed: int = 1,
                  chunk_tiles: int = 1024) -> Coo:
    """n x n matrix tiled tile x tile; each tile occupied with probability p.
    Occupied tiles draw their density from the mixture 20% dense (each entry
    present with probability 0.9), 30% bitmap-range (density U[0.15, 0.5]) and
    50% sparse (1-8 nnz placed uniformly).  Values N(0,1)."""
    rng = np.random.default_rng(seed)
    nb = (n + tile - 1) // tile
    total = nb * nb
    n_occ = int(rng.binomial(total, p))
    tiles = np.unique(rng.integers(0, total, size=n_occ, dtype=np.int64))
    kind = rng.random(tiles.size)
    dens = np.where(kind < 0.2, 0.9, rng.uniform(0.15, 0.5, size=tiles.size))
    sparse = kind >= 0.5
    tt = tile * tile
    rows_l, cols_l = [], []
    # dense / bitmap-range tiles: Bernoulli(density) per entry, in chunks
    dtiles = np.nonzero(~sparse)[0]
    for c0 in range(0, dtiles.size, chunk_tiles):
        sel = dtiles[c0:c0 + chunk_tiles]
        u = rng.random((sel.size, tt), dtype=np.float32)
        hit = u < dens[sel, None].astype(np.float32)
        ti, loc = np.nonzero(hit)
        tid = tiles[sel][ti]
        rows_l.append((tid // nb) * tile + loc // tile)
        cols_l.append((tid % nb) * tile + loc % tile)
    # sparse tiles: k in [1, 8] distinct positions
    stiles = np.nonzero(sparse)[0]
    ks = rng.integers(1, 9, size=stiles.size)
    locs = [rng.choice(tt, size=int(k), replace=False) for k in ks]
    if stiles.size:
        loc = np.concatenate(locs).astype(np.int64)
        tid = np.repeat(tiles[stiles], ks)
        rows_l.append((tid // nb) * tile + loc // tile)
        cols_l.append((tid % nb) * tile + loc % tile)
    rows = np.concatenate(rows_l).astype(np.int64)
    cols = np.concatenate(cols_l).astype(np.int64)
    keep = (rows < n) & (cols < n)
    rows, cols = rows[keep], cols[keep]
    vals = rng.standard_normal(rows.size)
    return Coo(rows, cols, vals, n, n, f"tiled_mixture_{n}_s{seed}")


def random_uniform(m: int, n: int, nnz: int, seed: int = 0, values: str = "normal") -> Coo:
    """nnz distinct positions uniformly at random (unsorted), values N(0,1)."""
    rng = np.random.default_rng(seed)
    nnz = min(nnz, m * n)
    keys = np.unique(rng.integers(0, m * n, size=int(nnz * 1.2) + 8, dtype=np.int64))
    keys = rng.permutation(keys)[:nnz]
    vals = rng.standard_normal(keys.size) if values == "normal" else np.ones(keys.size)
    return Coo(keys // n, keys % n, vals, m, n, f"random_{m}x{n}_{nnz}_s{seed}")


def random_blocky(m: int, n: int, s: int, n_tiles: int, seed: int = 0) -> Coo:
    """Tiles with densities spread over the whole COO/CSR/bitmap/dense range,
    so that every scheme is exercised at block size s."""
    rng = np.random.default_rng(seed)
    M, N = (m + s - 1) // s, (n + s - 1) // s
    tiles = np.unique(rng.integers(0, M * N, size=n_tiles, dtype=np.int64))
    rows_l, cols_l = [], []
    for t in tiles:
        d = rng.choice([0.002, 0.02, 0.08, 0.3, 0.7, 0.995, 1.0])
        hit = np.nonzero(rng.random(s * s) < d)[0]
        if hit.size == 0:
            hit = rng.integers(0, s * s, size=1)
        r = (t // N) * s + hit // s
        c = (t % N) * s + hit % s
        ok = (r < m) & (c < n)
        rows_l.append(r[ok])
        cols_l.append(c[ok])
    rows = np.concatenate(rows_l).astype(np.int64)
    cols = np.concatenate(cols_l).astype(np.int64)
    perm = rng.permutation(rows.size)
    return Coo(rows[perm], cols[perm], rng.standard_normal(rows.size), m, n,
               f"blocky_{m}x{n}_s{s}_seed{seed}")


def edge_shapes(n: int = 1000) -> list[Coo]:
    """The reference's pathological shapes (include/abhsf/utils/synthetic.h:8-91),
    seeded, at small size, plus ragged edges and a 1x1 matrix."""
    out = []
    i = np.arange(n, dtype=np.int64)
    one = np.ones(n)
    out.append(Coo(i, i, one.copy(), n, n, "diagonal"))
    out.append(Coo(i, np.zeros(n, dtype=np.int64), one.copy(), n, n, "single_column"))
    out.append(Coo(np.full(n, n - 1, dtype=np.int64), i, one.copy(), n, n, "single_row"))
    rr = np.concatenate([np.zeros(n, dtype=np.int64), i[1:]])
    cc = np.concatenate([i, np.zeros(n - 1, dtype=np.int64)])
    out.append(Coo(rr, cc, np.ones(rr.size), n, n, "single_row_column"))
    rng = np.random.default_rng(7)
    out.append(Coo(i, rng.integers(0, n, size=n), rng.standard_normal(n), n, n, "random_column"))
    d = 70
    dr, dc = np.divmod(np.arange(d * d, dtype=np.int64), d)
    out.append(Coo(dr, dc, rng.standard_normal(d * d), d, d, "dense_70"))
    out.append(Coo(np.array([0], dtype=np.int64), np.array([0], dtype=np.int64), np.array([2.5]), 1, 1, "one_by_one"))
    # ragged rectangular, empty rows and columns
    m2, n2 = 333, 517
    k = rng.choice(m2 * n2, size=4000, replace=False)
    keep = (k // n2) % 7 != 3
    k = k[keep]
    out.append(Coo(k // n2, k % n2, rng.standard_normal(k.size), m2, n2, "ragged_empty_rows"))
    return out


BLOCKGEN_SEED = 0x0498BC04  # the reference generator's seed (spmv/orig/88.cpp:46)


def block_pattern(bnnz: int = 1, kind: str = "random", block: int = 8, seed: int = BLOCKGEN_SEED) -> np.ndarray:
    """The (row, col) positions of one block as the reference's
    block_generator forms them (spmv/orig/88.cpp:43-141), sorted row-major
    (its std::set order, which finalize walks): "random" draws (row, col)
    pairs uniformly over the block until bnnz distinct ones are held
    (generate_random, 48-68); "diagonal", "single_row" and "single_col" are
    generate_diagonal / _single_row / _single_col (70-95).  The random draws
    come from numpy's PCG64 with the reference's seed, not from std::mt19937
    through std::uniform_int_distribution (whose mapping differs between
    standard-library versions): the same procedure and shape, another
    pattern."""
    if kind == "random":
        if not 0 < bnnz <= block * block:
            raise ValueError("bnnz must lie in 1 .. block * block")
        rng = np.random.default_rng(seed)
        held: set[tuple[int, int]] = set()
        while len(held) < bnnz:
            r, c = rng.integers(0, block, 2)
            held.add((int(r), int(c)))
        pos = sorted(held)
    elif kind == "diagonal":
        pos = [(k, k) for k in range(block)]
    elif kind == "single_row":
        pos = [(0, k) for k in range(block)]
    elif kind == "single_col":
        pos = [(k, 0) for k in range(block)]
    else:
        raise ValueError("kind: random, diagonal, single_row or single_col")
    return np.array(pos, dtype=np.int64).reshape(-1, 2)


def identical_blocks(num_blocks: int, bnnz: int = 1, kind: str = "random", block: int = 8,
                     seed: int = BLOCKGEN_SEED) -> Coo:
    """The reference's per-scheme block benchmark matrix (spmv/orig/88.cpp:716-840,
    4096 x 4096 blocks there): num_blocks x num_blocks copies of one block
    pattern (block_pattern), every value 1.0, elements in row order.  With
    x = 1 every SpMV adds bnnz * num_blocks^2 to the sum of y, the known
    answer the reference prints as its "y-vector sum"."""
    pat = block_pattern(bnnz, kind, block, seed)
    nb = int(num_blocks)
    # rows: block row I, pattern row; within a row, block columns J then pattern columns
    br = np.arange(nb, dtype=np.int64)
    rows_l, cols_l = [], []
    for pr in range(block):
        pc = pat[pat[:, 0] == pr, 1]
        if pc.size == 0:
            continue
        cols_one_row = (br[:, None] * block + pc[None, :]).reshape(-1)  # J-major, then pattern column
        rows_l.append((br * block + pr)[:, None].repeat(cols_one_row.size, axis=1))
        cols_l.append(np.broadcast_to(cols_one_row, (nb, cols_one_row.size)))
    rows = np.concatenate([r.reshape(-1) for r in rows_l])
    cols = np.concatenate([c.reshape(-1) for c in cols_l])
    order = np.lexsort((cols, rows))
    rows, cols = rows[order], cols[order]
    n = nb * block
    return Coo(rows, cols, np.ones(rows.size), n, n, f"identical_blocks_{nb}_{kind}_{pat.shape[0]}")


def banded(n: int, bandwidth: int, seed: int = 0) -> Coo:
    """Every entry within `bandwidth` of the diagonal (|i - j| <= bandwidth),
    values N(0,1): the banded half of the batched workload."""
    rng = np.random.default_rng(seed)
    offs = np.arange(-bandwidth, bandwidth + 1, dtype=np.int64)
    rows = np.repeat(np.arange(n, dtype=np.int64), offs.size)
    cols = rows + np.tile(offs, n)
    ok = (cols >= 0) & (cols < n)
    rows, cols = rows[ok], cols[ok]
    return Coo(rows, cols, rng.standard_normal(rows.size), n, n, f"banded_{n}_bw{bandwidth}_s{seed}")


def rmat(n: int, edge_factor: int = 8, a: float = 0.57, b: float = 0.19, c: float = 0.19, seed: int = 0) -> Coo:
    """R-MAT graph on n vertices: edge_factor * n edges, each placed by
    recursive quadrant choice with probabilities (a, b, c, 1 - a - b - c) on
    the 2^k x 2^k grid that covers n, those outside n x n dropped, duplicates
    merged; values N(0,1)."""
    rng = np.random.default_rng(seed)
    k = max(1, int(np.ceil(np.log2(max(n, 2)))))
    e = edge_factor * n
    r = np.zeros(e, dtype=np.int64)
    col = np.zeros(e, dtype=np.int64)
    for level in range(k):
        u = rng.random(e)
        bit = np.int64(1) << (k - 1 - level)
        r += np.where(u >= a + b, bit, 0)                      # quadrants c, d: lower half
        col += np.where(((u >= a) & (u < a + b)) | (u >= a + b + c), bit, 0)  # quadrants b, d: right half
    ok = (r < n) & (col < n)
    key = np.unique(r[ok] * n + col[ok])
    return Coo(key // n, key % n, rng.standard_normal(key.size), n, n, f"rmat_{n}_ef{edge_factor}_s{seed}")


def batched_set(count: int = 256, n_min: int = 1000, n_max: int = 200000, seed: int = 0):
    """The batched workload: count matrices, n log-uniform in [n_min, n_max];
    even ones banded (bandwidth U[3, 64]), odd ones R-MAT(0.57, 0.19, 0.19)
    with edge factor 8.  Yields the matrices one at a time."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_min), np.log(n_max), count)).astype(np.int64)
    bws = rng.integers(3, 65, count)
    for i in range(count):
        if i % 2 == 0:
            yield banded(int(ns[i]), int(bws[i]), seed=seed * 100003 + i)
        else:
            yield rmat(int(ns[i]), 8, seed=seed * 100003 + i)


def batched_set_device(count: int = 256, n_min: int = 1000, n_max: int = 200000, seed: int = 0, device="cuda"):
    """The batched workload generated on the GPU (torch's seeded Philox
    generator; the same distributions as batched_set, other random streams):
    yields (rows, cols, vals, m, n, name) with int64 / float64 CUDA tensors."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_min), np.log(n_max), count)).astype(np.int64)
    bws = rng.integers(3, 65, count)
    for i in range(count):
        n = int(ns[i])
        if i % 2 == 0:
            bw = int(bws[i])
            offs = torch.arange(-bw, bw + 1, device=device, dtype=torch.int64)
            rows = torch.arange(n, device=device, dtype=torch.int64).repeat_interleave(offs.numel())
            cols = rows + offs.repeat(n)
            ok = (cols >= 0) & (cols < n)
            rows, cols = rows[ok], cols[ok]
            name = f"banded_{n}_bw{bw}"
        else:
            k = max(1, int(np.ceil(np.log2(max(n, 2)))))
            e = 8 * n
            r = torch.zeros(e, device=device, dtype=torch.int64)
            c = torch.zeros(e, device=device, dtype=torch.int64)
            for level in range(k):
                u = torch.rand(e, device=device, generator=g, dtype=torch.float64)
                bit = 1 << (k - 1 - level)
                r += (u >= 0.76).to(torch.int64) * bit
                c += (((u >= 0.57) & (u < 0.76)) | (u >= 0.95)).to(torch.int64) * bit
            ok = (r < n) & (c < n)
            key = torch.unique(r[ok] * n + c[ok])
            rows, cols = key // n, key % n
            name = f"rmat_{n}_ef8"
        vals = torch.randn(rows.numel(), device=device, generator=g, dtype=torch.float64)
        yield rows, cols, vals, n, n, name


def rmat_device(scale: int = 22, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
                seed: int = 0, device="cuda"):
    """R-MAT graph on n = 2^scale vertices generated with torch on `device`
    (the distribution of rmat(); torch's seeded generator, so other random
    streams): edge_factor * n edges before duplicates are merged, values
    N(0,1).  Returns (rows, cols, vals, n) tensors sorted by row then column."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    n = 1 << scale
    e = edge_factor * n
    r = torch.zeros(e, device=device, dtype=torch.int64)
    col = torch.zeros(e, device=device, dtype=torch.int64)
    for level in range(scale):
        u = torch.rand(e, device=device, generator=g, dtype=torch.float64)
        bit = 1 << (scale - 1 - level)
        r += (u >= a + b).to(torch.int64) * bit
        col += (((u >= a) & (u < a + b)) | (u >= a + b + c)).to(torch.int64) * bit
    key = torch.unique(r * n + col)
    del r, col
    vals = torch.randn(key.numel(), device=device, generator=g, dtype=torch.float64)
    return key // n, key % n, vals, n


SELECTOR_FAMILIES = ("banded", "block_diagonal", "rmat", "stencil_2d", "stencil_3d")


def selector_matrix(seed: int, n_min: int = 10_000, n_max: int = 4_000_000, nnz_max: int = 16_000_000,
                    device="cuda"):
    """One matrix of the block-size selector's workload, generated with torch
    on `device` (Philox on CUDA; the CPU generator gives other matrices):
    family seed % 5 of SELECTOR_FAMILIES, n log-uniform in [n_min, n_max]
    (lowered so that the candidate entries stay within nnz_max), structure
    parameters drawn from numpy's default_rng(seed):

    banded          |i - j| <= w, w log-uniform [1, 300], each entry kept with
                    probability U[0.2, 1] (the diagonal always)
    block_diagonal  b x b diagonal blocks, b log-uniform [2, 512], fill U[0.05, 1]
    rmat            R-MAT with a U[0.45, 0.65], b = c = d = (1 - a) / 3, edge
                    factor log-uniform [2, 32], duplicates merged
    stencil_2d      5- or 9-point stencil on a g1 x g2 grid, g1 / g2 in [1/4, 4]
    stencil_3d      7- or 27-point stencil on a g1 x g2 x g3 grid

    Returns (rows, cols, m, n, name): int64 tensors on `device`, sorted by
    row then column."""
    import torch
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    fam = SELECTOR_FAMILIES[seed % len(SELECTOR_FAMILIES)]
    n = int(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
    i64 = dict(device=device, dtype=torch.int64)

    def keep(rows, cols, p):
        u = torch.rand(rows.numel(), device=device, generator=g)
        ok = (u < p) | (rows == cols)
        return rows[ok], cols[ok]

    if fam == "banded":
        w = int(round(np.exp(rng.uniform(0.0, np.log(300.0)))))
        p = float(rng.uniform(0.2, 1.0))
        n = max(n_min // 4, min(n, nnz_max // (2 * w + 1)))
        offs = torch.arange(-w, w + 1, **i64)
        rows = torch.arange(n, **i64).repeat_interleave(offs.numel())
        cols = rows + offs.repeat(n)
        ok = (cols >= 0) & (cols < n)
        rows, cols = keep(rows[ok], cols[ok], p)
        name = f"banded_n{n}_w{w}_p{p:.2f}"
    elif fam == "block_diagonal":
        b = int(round(np.exp(rng.uniform(np.log(2.0), np.log(512.0)))))
        p = float(rng.uniform(0.05, 1.0))
        n = max(n_min // 4, min(n, nnz_max // b))
        loc = torch.arange(b * b, **i64)
        base = torch.arange(0, n, b, **i64)
        rows = (base[:, None] + loc[None, :] // b).reshape(-1)
        cols = (base[:, None] + loc[None, :] % b).reshape(-1)
        ok = (rows < n) & (cols < n)
        rows, cols = keep(rows[ok], cols[ok], p)
        name = f"block_diagonal_n{n}_b{b}_p{p:.2f}"
    elif fam == "rmat":
        a = float(rng.uniform(0.45, 0.65))
        q = (1.0 - a) / 3.0
        ef = int(round(np.exp(rng.uniform(np.log(2.0), np.log(32.0)))))
        n = max(n_min // 4, min(n, nnz_max // ef))
        k = max(1, int(np.ceil(np.log2(max(n, 2)))))
        e = ef * n
        r = torch.zeros(e, **i64)
        c = torch.zeros(e, **i64)
        for level in range(k):
            u = torch.rand(e, device=device, generator=g, dtype=torch.float64)
            bit = 1 << (k - 1 - level)
            r += (u >= a + q).to(torch.int64) * bit
            c += (((u >= a) & (u < a + q)) | (u >= a + 2 * q)).to(torch.int64) * bit
        ok = (r < n) & (c < n)
        key = torch.unique(r[ok] * n + c[ok])
        rows, cols = key // n, key % n
        name = f"rmat_n{n}_a{a:.2f}_ef{ef}"
    else:
        d = 2 if fam == "stencil_2d" else 3
        wide = bool(rng.integers(0, 2))
        pts = (9 if wide else 5) if d == 2 else (27 if wide else 7)
        n = max(n_min // 4, min(n, nnz_max // pts))
        ratio = np.exp(rng.uniform(np.log(0.25), np.log(4.0), d - 1))
        side = n ** (1.0 / d)
        dims = [max(2, int(round(side * r))) for r in ratio]
        dims.append(max(2, n // int(np.prod(dims))))
        n = int(np.prod(dims))
        if wide:
            offs = np.array(np.meshgrid(*[[-1, 0, 1]] * d, indexing="ij")).reshape(d, -1).T
        else:
            offs = np.vstack([np.zeros(d, np.int64)] + [s * np.eye(d, dtype=np.int64)[k]
                                                        for k in range(d) for s in (-1, 1)])
        coord = torch.arange(n, **i64)
        idx = []
        rem = coord
        for size in dims[::-1]:
            idx.append(rem % size)
            rem = rem // size
        idx = idx[::-1]  # idx[k]: coordinate along dims[k], the last varying fastest
        stride = np.cumprod([1] + dims[::-1])[:-1][::-1]
        rl, cl = [], []
        for off in offs:
            ok = torch.ones(n, device=device, dtype=torch.bool)
            shift = 0
            for k in range(d):
                t = idx[k] + int(off[k])
                ok &= (t >= 0) & (t < dims[k])
                shift += int(off[k]) * int(stride[k])
            rl.append(coord[ok])
            cl.append(coord[ok] + shift)
        rows, cols = torch.cat(rl), torch.cat(cl)
        name = f"{fam}_{'x'.join(map(str, dims))}_{pts}pt"
    key = torch.sort(rows * n + cols).values
    return key // n, key % n, n, n, name


def rhs(n: int, seed: int = 0) -> np.ndarray:
    """x uniform[-1, 1]."""
    return np.random.default_rng(seed).uniform(-1.0, 1.0, size=n)
