"""CPU restatement of the block-size selector's arithmetic: the min-bss sweep,
the selector's features and the MLP's forward pass, gradients and Adam step,
all in float64 numpy.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the GPU
kernels, never by the product path.

min-bss follows block_statistics/min-bss.cpp:14-58 (least abhsf storage of the
mmf line over block sizes) over the square sizes 16..256, through this
oracle's own histograms and mmf lines (oracle.block_histogram, oracle.mmf_line,
themselves pinned against the reference's block_stats and mmf output).  The
row-nnz stdev feature is the population stdev of block_statistics/rows-nnz-stdev.cpp:11-30.
The features and the network have no counterpart in the reference.
"""
from __future__ import annotations

import numpy as np

from . import oracle

F, H, NC = 12, 64, 5
P = F * H + H + H * H + H + H * NC + NC + 2 * F
OW1 = 0
OB1 = OW1 + F * H
OW2 = OB1 + H
OB2 = OW2 + H * H
OW3 = OB2 + H
OB3 = OW3 + H * NC
OMEAN = OB3 + NC
OISTD = OMEAN + F
SIZES = (16, 32, 64, 128, 256)


def block_size_storage(rows, cols, m, n, mtype=oracle.TYPE_REAL, allow_csr=True):
    """abhsf (allow_csr) or abhsf134 bits of the mmf-double line at square
    sizes 16..256, and the size of least storage (ties to the smaller)."""
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    bits = []
    for k, s in enumerate(SIZES):
        hist = oracle.block_histogram(rows, cols, 4 + k, 4 + k)
        _, o2 = oracle.mmf_line(m, n, rows.size, mtype, s, s, hist)
        bits.append(o2[6] if allow_csr else o2[7])
    bits = np.array(bits, np.uint64)
    return bits, SIZES[int(np.argmin(bits))]


def features(rows, cols, m, n) -> np.ndarray:
    """The 12 selector features (float64) in the order of abhsf_selector_features."""
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    nnz = rows.size
    count = np.bincount(rows, minlength=m).astype(np.float64)
    mean = nnz / m
    std = np.sqrt(((count - mean) ** 2).sum() / m)
    d = np.abs(rows - cols)
    mn = max(m, n)
    hist = oracle.block_histogram(rows, cols, 6, 6)
    share = np.zeros(5)
    for z, c in hist.items():
        k = 0 if z <= 4 else 1 if z <= 32 else 2 if z <= 256 else 3 if z <= 1024 else 4
        share[k] += z * c
    blocks = sum(hist.values())
    M64 = (m + 63) // 64
    dn = max(nnz, 1)
    return np.array([np.log2(m), np.log2(n), np.log2(mean + 1.0), np.log2(std + 1.0),
                     (d.max() if nnz else 0) / mn, d.sum() / dn / mn, *(share / dn),
                     np.log2(blocks / M64 + 1.0)])


def _unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OW1:OB1].reshape(F, H), p[OB1:OW2], p[OW2:OB2].reshape(H, H), p[OB2:OW3],
            p[OW3:OB3].reshape(H, NC), p[OB3:OMEAN], p[OMEAN:OISTD], p[OISTD:OISTD + F])


def forward(p, X):
    """(probs, (xn, z1, h1, z2, h2)) of the network at rows of X."""
    W1, b1, W2, b2, W3, b3, mean, istd = _unpack(p)
    xn = (np.asarray(X, np.float64) - mean) * istd
    z1 = xn @ W1 + b1
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ W2 + b2
    h2 = np.maximum(z2, 0.0)
    lg = h2 @ W3 + b3
    lg = lg - lg.max(axis=1, keepdims=True)
    e = np.exp(lg)
    return e / e.sum(axis=1, keepdims=True), (xn, z1, h1, z2, h2)


def loss(p, X, T) -> float:
    """Mean cross-entropy against target distributions T."""
    probs, _ = forward(p, X)
    return float(-(np.asarray(T) * np.log(np.maximum(probs, 1e-300))).sum() / len(X))


def backward(p, X, T):
    """(gradient of the mean cross-entropy over all P parameters, zero on the
    normalisation entries; the loss)."""
    W1, b1, W2, b2, W3, b3, mean, istd = _unpack(p)
    probs, (xn, z1, h1, z2, h2) = forward(p, X)
    B = len(X)
    dl = (probs - np.asarray(T, np.float64)) / B
    d2 = (dl @ W3.T) * (h2 > 0)
    d1 = (d2 @ W2.T) * (h1 > 0)
    g = np.zeros(P)
    g[OW1:OB1] = (xn.T @ d1).reshape(-1)
    g[OB1:OW2] = d1.sum(axis=0)
    g[OW2:OB2] = (h1.T @ d2).reshape(-1)
    g[OB2:OW3] = d2.sum(axis=0)
    g[OW3:OB3] = (h2.T @ dl).reshape(-1)
    g[OB3:OMEAN] = dl.sum(axis=0)
    return g, loss(p, X, T)


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One bias-corrected Adam step of the trainable entries (all but the
    normalisation); returns new (p, m, v)."""
    p, g, m, v = (np.array(a, np.float64) for a in (p, g, m, v))
    t = slice(0, OMEAN)
    m[t] = b1 * m[t] + (1 - b1) * g[t]
    v[t] = b2 * v[t] + (1 - b2) * g[t] ** 2
    p[t] -= lr * (m[t] / (1 - b1 ** step)) / (np.sqrt(v[t] / (1 - b2 ** step)) + eps)
    return p, m, v
