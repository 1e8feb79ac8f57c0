"""Regenerates the golden fixtures in this directory by running the reference's
own programs, compiled from the reference sources by ``make -C oracle ref``:

* ``oracle/_ref/block_stats`` (block_statistics/block_stats.cpp) -> ``props``
  and the 64 ``RxS.bstats`` block histograms;
* ``oracle/_ref/mmf`` (block_statistics/mmf.cpp) -> ``mmf-single`` and
  ``mmf-double`` minimum-storage totals;
* ``oracle/_ref/libref_csr.so`` (csr_matrix::spmv_naive,
  spmv/bottlenecks/spmv.cpp:58-64) -> y += A x for seeded x and y.

Needs the reference tree (REF, default: a "reference" directory beside the repository) and is run by hand in
the development container; the fixtures it writes are committed, so nothing
at test time reads the reference.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from abhsf_b200 import workloads as W  # noqa: E402
from oracle import oracle  # noqa: E402

REF = os.environ.get("REF") or os.path.join(os.path.dirname(ROOT), "reference")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def write_mtx(path, coo: W.Coo, field="real", symmetry="general"):
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {field} {symmetry}\n")
        f.write(f"{coo.m} {coo.n} {coo.nnz}\n")
        r = coo.rows + 1
        c = coo.cols + 1
        if field == "pattern":
            np.savetxt(f, np.stack([r, c], 1), fmt="%d %d")
        elif field == "integer":
            np.savetxt(f, np.stack([r, c, coo.vals.astype(np.int64)], 1), fmt="%d %d %d")
        else:
            for a, b, v in zip(r.tolist(), c.tolist(), coo.vals.tolist()):
                f.write(f"{a} {b} {v!r}\n")


def read_mtx(path) -> W.Coo:
    rows, cols, vals = [], [], []
    with open(path) as f:
        header = f.readline()
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        m, n, _ = (int(t) for t in line.split())
        for line in f:
            t = line.split()
            if not t:
                continue
            rows.append(int(t[0]) - 1)
            cols.append(int(t[1]) - 1)
            vals.append(float(t[2]) if len(t) > 2 else 1.0)
    assert "coordinate" in header
    return W.Coo(np.array(rows, dtype=np.int64), np.array(cols, dtype=np.int64),
                 np.array(vals, dtype=np.float64), m, n)


def run_reference_stats(mtx_path: str, props_type: int | None = None) -> dict:
    """block_stats + mmf on one .mtx.  props_type rewrites the type field of
    ``props`` before mmf runs: block_stats drops every element of a pattern or
    integer matrix (block_stats.cpp:46 reads only the real value slot, which
    the reader leaves 0.0 for those types, and block_stats.cpp:53 discards
    zeros, then asserts on the empty set).  mmf's binary and integer paths
    (mmf.cpp:32-47,77-80) are therefore pinned by running block_stats on the
    real-valued copy and mmf with the type rewritten."""
    d = tempfile.mkdtemp(prefix="abhsf_golden_")
    subprocess.run([os.path.join(REF_DIR, "block_stats"), os.path.abspath(mtx_path)], cwd=d,
                   check=True, stdout=subprocess.DEVNULL)
    if props_type is not None:
        t = open(os.path.join(d, "props")).read().split()
        t[5] = str(props_type)
        open(os.path.join(d, "props"), "w").write(" ".join(t) + "\n")
    subprocess.run([os.path.join(REF_DIR, "mmf")], cwd=d, check=True, stdout=subprocess.DEVNULL)
    out = {"props": [int(t) for t in open(os.path.join(d, "props")).read().split()], "bstats": {}}
    for k in range(1, 9):
        for l in range(1, 9):
            name = f"{1 << k}x{1 << l}"
            hist = {}
            for line in open(os.path.join(d, name + ".bstats")):
                z, c = line.split()
                hist[z] = int(c)
            out["bstats"][name] = hist
    for prec in ("single", "double"):
        out["mmf_" + prec] = [[int(t) for t in line.split()]
                              for line in open(os.path.join(d, "mmf-" + prec)) if line.strip()]
    subprocess.run(["rm", "-rf", d], check=True)
    return out


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all", "ref", f"REF={REF}"], check=True)
    work = tempfile.mkdtemp(prefix="abhsf_mtx_")

    small: dict[str, tuple[W.Coo, str, str]] = {}
    tm = read_mtx(os.path.join(REF, "block_statistics", "experiments", "test.mtx"))
    tm.name = "test_mtx"
    small["test_mtx"] = (tm, "real", "general")
    small["rand_real"] = (W.random_uniform(300, 517, 5000, seed=3), "real", "general")
    pat = W.random_uniform(400, 400, 3000, seed=4, values="ones")
    small["rand_pattern"] = (pat, "pattern", "general")
    ri = W.random_uniform(250, 260, 2000, seed=6)
    ri.vals = np.round(ri.vals * 10)
    ri.vals[ri.vals == 0] = 3.0
    small["rand_integer"] = (ri, "integer", "general")
    sl = W.random_uniform(300, 300, 2500, seed=8)
    lower = sl.rows >= sl.cols
    small["sym_lower"] = (W.Coo(sl.rows[lower], sl.cols[lower], sl.vals[lower], 300, 300), "real", "symmetric")
    small["blocky64"] = (W.random_blocky(500, 700, 64, 60, seed=5), "real", "general")
    small["blocky16"] = (W.random_blocky(130, 150, 16, 60, seed=9), "real", "general")
    for e in W.edge_shapes(300):
        if e.name in ("diagonal", "single_row_column", "dense_70", "ragged_empty_rows", "one_by_one"):
            small["edge_" + e.name] = (e, "real", "general")

    stats = {}
    arrays = {}
    spmv = {}
    for name, (coo, field, sym) in small.items():
        p = os.path.join(work, name + ".mtx")
        if field in ("pattern", "integer"):
            write_mtx(p, coo, "real", sym)
            stats[name] = run_reference_stats(p, props_type=0 if field == "pattern" else 1)
        else:
            write_mtx(p, coo, field, sym)
            stats[name] = run_reference_stats(p)
        stats[name]["field"] = field
        stats[name]["symmetry"] = sym
        arrays[name + "__rows"] = coo.rows
        arrays[name + "__cols"] = coo.cols
        arrays[name + "__vals"] = coo.vals
        arrays[name + "__shape"] = np.array([coo.m, coo.n], dtype=np.int64)
        if field == "real" and sym == "general":
            rng = np.random.default_rng(100 + len(spmv))
            x = rng.uniform(-1, 1, coo.n)
            y0 = rng.uniform(-1, 1, coo.m)
            y = y0.copy()
            ref = oracle.RefCSR(coo.rows, coo.cols, coo.vals, coo.m, coo.n)
            ref.spmv(x, y)
            ref.release()
            spmv[name + "__x"] = x
            spmv[name + "__y0"] = y0
            spmv[name + "__y"] = y

    c1 = W.laplacian_2d(512)
    p = os.path.join(work, "laplace2d_512.mtx")
    write_mtx(p, c1)
    stats["laplace2d_512"] = run_reference_stats(p)
    stats["laplace2d_512"]["field"] = "real"
    stats["laplace2d_512"]["symmetry"] = "general"
    # reference CSR y on the 512 x 512 2D Laplacian with x from seed 0 (stored as a checksum set:
    # the full vector is regenerated at test time and compared through these)
    x = W.rhs(c1.n, seed=0)
    y = np.zeros(c1.m)
    ref = oracle.RefCSR(c1.rows, c1.cols, c1.vals, c1.m, c1.n)
    ref.spmv(x, y)
    ref.release()
    spmv["laplace2d_512__y_seed0"] = y

    with open(os.path.join(HERE, "block_stats.json"), "w") as f:
        json.dump(stats, f, indent=0, sort_keys=True)
    np.savez_compressed(os.path.join(HERE, "matrices.npz"), **arrays)
    np.savez_compressed(os.path.join(HERE, "spmv_ref.npz"), **spmv)
    subprocess.run(["rm", "-rf", work], check=True)
    print("wrote", sorted(stats))


if __name__ == "__main__":
    main()
