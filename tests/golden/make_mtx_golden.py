"""Writes the Matrix Market fixtures in tests/golden/mtx/ and records what the
reference's own reader, read_mtx_real_or_binary
(include/abhsf/utils/matrix_market_reader.h:146-200, compiled from the
reference sources by `make -C oracle ref` into oracle/_ref/libref_mtx.so),
reads from each: tests/golden/mtx_ref.npz.  Run by hand in the development
container; the fixtures are committed, so nothing at test time reads the
reference.

    python tests/golden/make_mtx_golden.py
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
MTX = os.path.join(HERE, "mtx")
LIB = os.path.join(ROOT, "oracle", "_ref", "libref_mtx.so")


def fixtures() -> dict[str, str]:
    """name -> file text."""
    rng = np.random.default_rng(11)
    f = {}
    f["real_general"] = (
        "%%MatrixMarket matrix coordinate real general\n"
        "% a comment line\n%\n"
        "5 6 9\n"
        "1 1 1.5\n2 3 -2e-3\n3 4 0\n3 1 .25\n1 6 7\n"
        "5 5 1.0000000000000002\n4 2 3.141592653589793238462643\n2 2 -0.0\n5 1 4.9e-324\n")
    f["pattern_general"] = (
        "%%MatrixMarket matrix coordinate pattern general\n4 4 5\n1 2\n2 1\n3 3\n4 1\n4 4\n")
    f["real_symmetric_lower"] = (
        "%%MatrixMarket matrix coordinate real symmetric\n4 4 6\n1 1 2\n2 1 -1\n2 2 2\n3 2 -1\n4 3 -1\n4 4 2\n")
    f["pattern_symmetric_upper"] = (
        "%%MatrixMarket matrix coordinate pattern symmetric\n3 3 4\n1 1\n1 2\n2 3\n3 3\n")
    f["crlf_and_case"] = (
        "%%MatrixMarket Matrix Coordinate Real General\r\n3 3 3\r\n1 1 1e1\r\n2 2 -3.5\r\n3 1 1E-5\r\n")
    f["extra_lines_after_nnz"] = (
        "%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 1\n2 2 2\n3 3 3\n")
    # many values printed to 17 significant digits and to fewer: exact rounding
    m, n, k = 300, 280, 4000
    key = rng.choice(m * n, size=k, replace=False)
    vals = rng.standard_normal(k) * 10.0 ** rng.integers(-30, 30, k)
    lines = [f"{int(q // n) + 1} {int(q % n) + 1} {v:.17g}" if i % 2 else f"{int(q // n) + 1} {int(q % n) + 1} {v:.6e}"
             for i, (q, v) in enumerate(zip(key, vals))]
    f["random_real"] = "%%MatrixMarket matrix coordinate real general\n" + f"{m} {n} {k}\n" + "\n".join(lines) + "\n"
    return f


def main() -> None:
    L = C.CDLL(LIB)
    L.ref_mtx_read.restype = C.c_long
    L.ref_mtx_read.argtypes = [C.c_char_p, C.POINTER(C.c_long), C.POINTER(C.c_long), C.c_long,
                               C.c_void_p, C.c_void_p, C.c_void_p]
    os.makedirs(MTX, exist_ok=True)
    out = {}
    for name, text in fixtures().items():
        path = os.path.join(MTX, name + ".mtx")
        with open(path, "w", newline="") as fh:
            fh.write(text)
        cap = 1 << 16
        rows = np.zeros(cap, np.int64)
        cols = np.zeros(cap, np.int64)
        vals = np.zeros(cap, np.float64)
        m, n = C.c_long(), C.c_long()
        k = L.ref_mtx_read(path.encode(), C.byref(m), C.byref(n), cap, rows.ctypes.data, cols.ctypes.data,
                           vals.ctypes.data)
        assert k >= 0, (name, k)
        out[name + "__rows"] = rows[:k]
        out[name + "__cols"] = cols[:k]
        out[name + "__vals"] = vals[:k]
        out[name + "__shape"] = np.array([m.value, n.value])
    np.savez_compressed(os.path.join(HERE, "mtx_ref.npz"), **out)
    print("wrote", len(out) // 4, "fixtures")


if __name__ == "__main__":
    main()
