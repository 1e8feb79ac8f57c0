"""Throughput benchmark of the ABHSF FP64 SpMV hot path on B200.

Workload: the tiled-mixture matrix (n = 4,194,304, 64 x 64 tiles; 20% dense
0.9, 30% density U[0.15, 0.5], 50% 1-8 nnz; ~60M nnz; values N(0,1), x
U[-1, 1], seed 1), block size 64, scheme per tile by exact minimum storage.

A step is one y += A x over the whole matrix.  value = algorithmic bytes per
step / kernel time, where algorithmic bytes B = format bytes + 8 n (x read
once) + 16 m (y read and written).  e2e is the same metric through the
host-memory call (x, y in pinned host memory; copies inside the timed region).

Every further measurement (SpMM, the batch, low precision, CG, the other
matrix shapes, cuSPARSE, the selector, ...) is printed as a JSON line of its
own ({"section": name, ...}) before the headline line, which comes last.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU (torchrun): every rank runs an independent replica (the SpMV has no
exchange step); value is the bytes all ranks processed / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time
import warnings

import numpy as np

warnings.filterwarnings("ignore", message=".*[Ss]parse.*")  # torch's beta-state notes on CSR tensors

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SpMV GB/s (% HBM peak) + CG solve time, tuned vs plain on one B200 at same tol"
UNIT = "GB/s"
FALLBACK_HBM_GBS = 6650.0
L2_FLUSH_BYTES = 256 << 20
DEFAULT_N = 4_194_304
X_SEED = 1  # x U[-1, 1] of the timed matrix, in both arms
KERNELS = {"reference": "k_spmv_f64_ring", "tree": "k_spmv_f64"}


def traffic_file(sum_order):
    return os.path.join(ROOT, "profiles", f"{KERNELS[sum_order]}_tiled_mixture_n{DEFAULT_N}_s64.md")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic_per_launch(sum_order, n):
    """DRAM bytes (read + write) per SpMV launch from the committed ncu summary
    of this kernel on the default workload (None for other sizes)."""
    if n != DEFAULT_N:
        return None
    try:
        txt = open(traffic_file(sum_order)).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", txt)
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.proc = None
        self.idx = gpu_index
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(gpu_index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = [[t.strip() for t in line.split(",")] for line in out.strip().splitlines() if line.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def workload(args):
    """The timed matrix: the tiled mixture (default), or for profiling the 3D
    7-point Laplacian on a grid^3 mesh or R-MAT scale 22."""
    from abhsf_b200 import workloads as W
    t0 = time.time()
    if args.matrix == "laplacian3d":
        c = W.laplacian_3d(args.grid)
        c.name = f"laplacian3d g={args.grid} (7-point, diag 6, off -1)"
    elif args.matrix == "rmat22":
        rows, cols, vals, n = W.rmat_device(22, 16, seed=1, device="cuda")
        c = W.Coo(rows.cpu().numpy(), cols.cpu().numpy(), vals.cpu().numpy(), n, n, "rmat22")
        c.name = "R-MAT scale 22 (0.57, 0.19, 0.19), edge factor 16, values N(0,1)"
        del rows, cols, vals
    else:
        c = W.tiled_mixture(n=args.n)
        c.name = f"tiled_mixture n={c.n} tile=64 p=1.2266e-5 seed=1 (values N(0,1)), x U[-1,1] seed {X_SEED}"
    log(f"workload: {c.name} nnz={c.nnz} ({time.time() - t0:.1f} s to generate)")
    return c


def algorithmic_bytes(st: dict, m: int, n: int) -> int:
    return int(st["format_bytes"]) + 8 * n + 16 * m


def time_spmm(A, c, st, dev, stream, l2_flush, warmup, ks=(4, 8, 16, 32), steps=5):
    """Y += A X on the same matrix for a few k (X, Y row-major, resident in
    HBM); bytes per call B_fmt + k (8 n + 16 m), FLOPs 2 nnz k."""
    import torch
    out = {}
    for k in ks:
        X = torch.rand((c.n, k), dtype=torch.float64, device=dev)
        Y = torch.zeros((c.m, k), dtype=torch.float64, device=dev)
        for _ in range(max(warmup, 1)):
            l2_flush()
            A.spmm(X, Y)
        ts = []
        for _ in range(steps):
            l2_flush()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            A.spmm(X, Y)
            e1.record(stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        t = sum(ts) / len(ts)
        b = int(st["format_bytes"]) + k * (8 * c.n + 16 * c.m)
        out[str(k)] = {"ms": t, "GB/s": b / (t * 1e-3) / 1e9, "gflops": 2.0 * c.nnz * k / (t * 1e-3) / 1e9,
                       "bytes": b}
        del X, Y
    return out


def time_lowprec(c, dev, l2_flush, warmup, steps=10):
    """f32 and bf16 copies of the same matrix: f32 SpMV time, GB/s over what
    one SpMV reads (spmv_bytes + 4 n + 8 m) and error against an FP64 product
    of the same (f32) x computed apart from this library (torch's CSR SpMV,
    cuSPARSE, in FP64): normwise, and the largest |y - y64| / (|A| |x|) per
    element.  The same errors on R-MAT scale 22 (n = 4,194,304, edge factor
    16, values N(0,1))."""
    import torch
    from abhsf_b200 import AbhsfMatrix
    from abhsf_b200 import workloads as W

    def errors(rows, cols, vals, m, n, vt, x32):
        Acs = _csr_tensor(rows, cols, vals, m, n, dev)
        y64 = torch.mv(Acs, x32.double())
        Aabs = torch.sparse_csr_tensor(Acs.crow_indices(), Acs.col_indices(), Acs.values().abs(), size=(m, n))
        scale = torch.mv(Aabs, x32.double().abs())
        del Acs, Aabs
        A = AbhsfMatrix.from_elements(rows, cols, vals, m, n, block_size=64, value_type=vt)
        y = torch.zeros(m, dtype=torch.float32, device=dev)
        A.spmv_f32(x32, y)
        d = (y.double() - y64).abs()
        nz = scale > 0
        return A, y, {"rel_err_vs_fp64": float(torch.linalg.norm(y.double() - y64) / torch.linalg.norm(y64)),
                      "max_err_over_absAx": float((d[nz] / scale[nz]).max())}

    x32 = torch.rand(c.n, dtype=torch.float32, device=dev) * 2 - 1
    out = {}
    for vt in ("f32", "bf16"):
        A, y, err = errors(c.rows, c.cols, c.vals, c.m, c.n, vt, x32)
        for _ in range(max(warmup, 1)):
            l2_flush()
            A.spmv_f32(x32, y)
        ts = []
        for _ in range(steps):
            l2_flush()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            A.spmv_f32(x32, y)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        t = sum(ts) / len(ts)
        b = int(A.stats()["spmv_bytes"]) + 4 * c.n + 8 * c.m
        out[vt] = dict(err, ms=t, bytes=b, **{"GB/s": b / (t * 1e-3) / 1e9})
        A.release()
    rows, cols, vals, n = W.rmat_device(22, 16, seed=1, device=dev)
    x32 = torch.rand(n, dtype=torch.float32, device=dev) * 2 - 1
    out["rmat22"] = {"workload": f"R-MAT scale 22 edge factor 16 (0.57, 0.19, 0.19), nnz={rows.numel()}, "
                                 "values N(0,1), x U[-1,1] f32, block size 64",
                     "fp64_reference": "torch.mv on a CSR tensor (cuSPARSE), FP64"}
    for vt in ("f32", "bf16"):
        A, _, err = errors(rows, cols, vals, n, n, vt, x32)
        A.release()
        out["rmat22"][vt] = err
    del rows, cols, vals
    return out


def time_batched(dev, l2_flush, warmup, count=256, steps=10):
    """The batched workload (count matrices, n log-uniform [1k, 200k], half
    banded with bandwidth U[3, 64], half R-MAT(0.57, 0.19, 0.19) edge factor 8,
    values N(0,1), generated on the GPU), block size autotuned over the five
    sizes (the batched launch timed at each): all SpMVs as one launch
    (abhsf_batch_spmv) against one abhsf_spmv launch per matrix."""
    import torch
    from abhsf_b200 import AbhsfBatch, AbhsfMatrix
    from abhsf_b200 import workloads as W
    t0 = time.time()
    sets = {s: [] for s in (16, 32, 64, 128, 256)}
    byts = {s: 0 for s in sets}
    nnz = 0
    fbyts = {s: 0 for s in sets}
    for rows, cols, vals, m, n, _ in W.batched_set_device(count, seed=0, device=dev):
        for s in sets:
            A = AbhsfMatrix.from_elements(rows, cols, vals, m, n, block_size=s)
            sets[s].append(A)
            st_ = A.stats()
            byts[s] += int(st_["spmv_bytes"]) + 8 * n + 16 * m
            fbyts[s] += int(st_["format_bytes"]) + 8 * n + 16 * m
        nnz += int(rows.numel())
        del rows, cols, vals
    build_s = time.time() - t0
    xs = [torch.rand(A.n, dtype=torch.float64, device=dev) for A in sets[64]]
    ys = [torch.zeros(A.m, dtype=torch.float64, device=dev) for A in sets[64]]

    def timed(fn):
        for _ in range(max(warmup, 1)):
            l2_flush()
            fn()
        ts = []
        for _ in range(steps):
            l2_flush()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return sum(ts) / len(ts)

    # autotune the batch's block size: the one batched launch timed at each size
    tune = {}
    for s, ms_ in sets.items():
        b_ = AbhsfBatch(ms_)
        px_, py_ = b_.pointer_tables(xs, ys)
        tune[s] = timed(lambda: b_.spmv_tables(px_, py_))
        b_.release()
    s_best = min(tune, key=tune.get)
    mats = sets[s_best]
    byts = byts[s_best]
    fbyts = fbyts[s_best]
    batch = AbhsfBatch(mats)
    px, py = batch.pointer_tables(xs, ys)

    def one_by_one():
        for A, x, y in zip(mats, xs, ys):
            A.spmv(x, y)

    t_batch = timed(lambda: batch.spmv_tables(px, py))
    t_loop = timed(one_by_one)
    # spot check: matrix 0 through the batch equals its own SpMV
    y_a, y_b = ys[0].clone(), ys[0].clone()
    mats[0].spmv(xs[0], y_a)
    ys[0].copy_(y_b)
    batch.spmv_tables(px, py)
    torch.cuda.synchronize()
    same = bool(torch.equal(ys[0], y_a))
    if batch.status() != 0:
        raise RuntimeError("batched SpMV reported a device status")
    out = {"workload": f"{count} matrices, n log-uniform [1k, 200k], even banded (bandwidth U[3,64]), odd R-MAT"
                       f"(0.57, 0.19, 0.19) edge factor 8, values N(0,1), generated on the GPU",
           "block_size": s_best, "autotune_ms": {str(k): v for k, v in tune.items()},
           "nnz": nnz, "bytes_per_step": byts, "format_bytes_per_step": fbyts,
           "bytes_note": "what one SpMV of every matrix reads (spmv_bytes + 8 n + 16 m); format_bytes_per_step counts "
                         "the ABHSF arrays instead",
           "build_s": build_s,
           "batched": {"ms": t_batch, "GB/s": byts / (t_batch * 1e-3) / 1e9, "launches": batch.launches(),
                       "graph": "capturable (one graph node per launch)"},
           "one_by_one": {"ms": t_loop, "GB/s": byts / (t_loop * 1e-3) / 1e9, "launches": count},
           "speedup": t_loop / t_batch, "matrix0_bitwise": same}
    batch.release()
    for ms_ in sets.values():
        for A in ms_:
            A.release()
    return out


def time_cg(dev, g=256, rtol=1e-10):
    """CG solve time on the 3D 7-point Laplacian g^3 (n = g^3, SPD, b U[-1,1]
    seed 1, x0 = 0) to ||b - A x|| <= rtol ||b||: the plain form (FP64 CG,
    block size 64) against the tuned form: the block size the selector trained
    on measured SpMV time picks, and mixed precision -- f32 CG on an f32 or a bf16 copy, the
    solution, the residual replacement and the convergence test in FP64 --
    with every 8 iterations replayed as one CUDA graph.  (6 and -1 are exact
    in bf16, so the bf16 copy is the matrix itself.)"""
    import torch
    from abhsf_b200 import AbhsfMatrix, cg, cg_mixed
    from abhsf_b200 import selector as sel
    from abhsf_b200 import workloads as W
    lap = W.laplacian_3d(g)
    rows_d = torch.from_numpy(lap.rows).to(dev)
    cols_d = torch.from_numpy(lap.cols).to(dev)
    t0 = time.perf_counter()
    feats = sel.features(rows_d, cols_d, lap.m, lap.n)
    s_learned = sel.predict(feats, model=sel.builtin_time_model())  # trained on measured SpMV time
    t_select = time.perf_counter() - t0
    s_storage = sel.predict(feats)  # the storage-trained model's choice, for the record
    del rows_d, cols_d
    A64 = AbhsfMatrix.from_elements(lap.rows, lap.cols, lap.vals, lap.m, lap.n, block_size=64)
    L64 = AbhsfMatrix.from_elements(lap.rows, lap.cols, lap.vals, lap.m, lap.n, block_size=s_learned)
    L32 = AbhsfMatrix.from_elements(lap.rows, lap.cols, lap.vals, lap.m, lap.n, block_size=s_learned,
                                    value_type="f32")
    L16 = AbhsfMatrix.from_elements(lap.rows, lap.cols, lap.vals, lap.m, lap.n, block_size=s_learned,
                                    value_type="bf16")
    b = torch.from_numpy(np.random.default_rng(1).uniform(-1, 1, lap.n)).to(dev)
    out = {"workload": f"3D 7-point Laplacian {g}^3 (n={lap.n}, nnz={lap.nnz}, diag 6, off -1), b U[-1,1] seed 1, "
                       f"x0 = 0", "rtol": rtol, "learned_block_size": s_learned, "select_s": t_select,
           "selector": "learned_time (MLP trained on measured SpMV time)", "storage_model_block_size": s_storage}
    # each solver's SpMV alone (working set > L2; CUDA events, 10 launches after 3)
    peak, _ = hbm_peak()
    for key, M, dt in (("spmv_f64", A64, torch.float64), ("spmv_f32_copy", L32, torch.float32),
                       ("spmv_bf16_copy", L16, torch.float32)):
        xs = torch.rand(lap.n, dtype=dt, device=dev)
        ys = torch.zeros(lap.n, dtype=dt, device=dev)
        fn = (lambda: M.spmv(xs, ys)) if dt == torch.float64 else (lambda: M.spmv_f32(xs, ys))
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(10):
            fn()
        e1.record()
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 10
        es = 8 if dt == torch.float64 else 4
        byts = int(M.stats()["spmv_bytes"]) + es * lap.n + 2 * es * lap.n
        out[key] = {"ms": t, "GB/s": byts / (t * 1e-3) / 1e9, "frac_of_peak": byts / (t * 1e-3) / 1e9 / peak,
                    "bytes": byts, "block_size": M.block_size}
        del xs, ys
    # each solver twice from x0 = 0 (same iterations both times); the faster
    # solve is reported, both are listed, and the SM clocks are sampled
    clocks = ClockSampler(torch.cuda.current_device())
    for name, fn in (("plain", lambda x: cg(A64, b, x, rtol=rtol)),
                     ("tuned_f32", lambda x: cg_mixed(L64, L32, b, x, rtol=rtol, update_factor=0.1)),
                     ("tuned_bf16", lambda x: cg_mixed(L64, L16, b, x, rtol=rtol, update_factor=0.1))):
        runs = []
        for _ in range(2):
            x = torch.zeros(lap.n, dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            info = fn(x)
            torch.cuda.synchronize()
            runs.append(time.perf_counter() - t0)
        out[name] = dict(info, seconds=min(runs), runs_s=runs)
    out["clocks"] = clocks.stop()
    out["plain"]["solver"] = "FP64 CG, block size 64, reference-order f64 SpMV"
    out["tuned_f32"]["solver"] = (f"block size {s_learned} (time-trained selector): f32 CG on an f32 copy, FP64 "
                                  "solution, FP64 residual replacement each 10x drop")
    out["tuned_bf16"]["solver"] = out["tuned_f32"]["solver"].replace("an f32 copy", "a bf16 copy")
    out["tuned_f32_speedup"] = out["plain"]["seconds"] / out["tuned_f32"]["seconds"]
    out["tuned_bf16_speedup"] = out["plain"]["seconds"] / out["tuned_bf16"]["seconds"]
    for M in (A64, L64, L32, L16):
        M.release()
    return out


def time_cusparse(c, dev, l2_flush, warmup, ours_ms, steps=10):
    """A further reference point on the same GPU: cuSPARSE's CSR SpMV (through
    torch.mv on a CSR tensor, int32 indices, FP64 values) on the same matrix
    and x.  Its own CSR bytes are 12 nnz + 4 (m + 1) + 8 n + 8 m (y written,
    not read: it computes y = A x)."""
    import torch
    try:
        order = np.lexsort((c.cols, c.rows))
        crow = np.zeros(c.m + 1, np.int64)
        np.cumsum(np.bincount(c.rows, minlength=c.m), out=crow[1:])
        A = torch.sparse_csr_tensor(torch.from_numpy(crow.astype(np.int32)).to(dev),
                                    torch.from_numpy(c.cols[order].astype(np.int32)).to(dev),
                                    torch.from_numpy(c.vals[order]).to(dev), size=(c.m, c.n))
        x = torch.rand(c.n, dtype=torch.float64, device=dev) * 2 - 1
        for _ in range(max(warmup, 1)):
            l2_flush()
            y = torch.mv(A, x)
        ts = []
        for _ in range(steps):
            l2_flush()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            y = torch.mv(A, x)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        t = sum(ts) / len(ts)
        b = 12 * c.nnz + 4 * (c.m + 1) + 8 * c.n + 8 * c.m
        del A, y
        return {"ms": t, "GB/s_own_csr_bytes": b / (t * 1e-3) / 1e9, "csr_bytes": b,
                "gflops": 2.0 * c.nnz / (t * 1e-3) / 1e9, "ours_speedup": t / ours_ms,
                "call": "torch.mv(sparse_csr_tensor int32 indices, f64 values) -> cuSPARSE SpMV"}
    except Exception as e:  # a reference point only: report why it is missing
        return {"unavailable": f"{type(e).__name__}: {e}"[:300]}


def _events_time(fn, l2_flush, warmup, steps):
    """Mean CUDA-event time (ms) of fn on the current stream, L2 flushed
    before every call."""
    import torch
    for _ in range(max(warmup, 1)):
        l2_flush()
        fn()
    ts = []
    for _ in range(steps):
        l2_flush()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    return sum(ts) / len(ts)


def _csr_tensor(rows, cols, vals, m, n, dev):
    """torch CSR tensor (int32 indices, f64 values) of COO triplets on dev."""
    import torch
    rows = torch.as_tensor(rows, device=dev)
    cols = torch.as_tensor(cols, device=dev)
    vals = torch.as_tensor(vals, device=dev, dtype=torch.float64)
    order = torch.argsort(rows * n + cols)
    crow = torch.zeros(m + 1, dtype=torch.int64, device=dev)
    crow[1:] = torch.cumsum(torch.bincount(rows, minlength=m), 0)
    return torch.sparse_csr_tensor(crow.to(torch.int32), cols[order].to(torch.int32), vals[order], size=(m, n))


def time_shapes(dev, l2_flush, warmup, steps=10):
    """The named shapes beside the timed matrix: the 2D 5-point Laplacian
    512^2 (the reference's CPU-runnable configuration), the 3D 7-point
    Laplacian 256^3 and R-MAT scale 22 (edge factor 16, values N(0,1)), block
    size 64, the default build: FP64 SpMV time, GB/s over what one SpMV reads
    (spmv_bytes + 8 n + 16 m) and over the format bytes, the fraction of the
    measured copy peak, how much of the matrix is in row slices, and
    cuSPARSE's CSR SpMV (torch.mv, int32 indices) on the same matrix and GPU."""
    import torch
    from abhsf_b200 import AbhsfMatrix
    from abhsf_b200 import workloads as W
    peak, _ = hbm_peak()
    out = {}

    def one(name, rows, cols, vals, m, n, desc):
        A = AbhsfMatrix.from_elements(rows, cols, vals, m, n, block_size=64)
        st = A.stats()
        P = A.slices()
        x = torch.rand(n, dtype=torch.float64, device=dev) * 2 - 1
        y = torch.zeros(m, dtype=torch.float64, device=dev)
        ms = _events_time(lambda: A.spmv(x, y), l2_flush, warmup, steps)
        if A.device_status():
            raise RuntimeError(f"{name}: device status {A.device_status()}")
        A.release()
        b = int(st["spmv_bytes"]) + 8 * n + 16 * m
        bf = int(st["format_bytes"]) + 8 * n + 16 * m
        r = {"workload": desc, "nnz": int(st["nnz"]), "ms": ms, "GB/s": b / (ms * 1e-3) / 1e9,
             "frac_of_peak": b / (ms * 1e-3) / 1e9 / peak, "bytes": b, "format_bytes_per_step": bf,
             "gflops": 2.0 * st["nnz"] / (ms * 1e-3) / 1e9,
             "slice_elements": int(P["elements"]), "chains": int(P["chain"].sum()),
             "schemes": st["tiles_per_scheme"]}
        try:
            Acs = _csr_tensor(rows, cols, vals, m, n, dev)
            ms_c = _events_time(lambda: torch.mv(Acs, x), l2_flush, warmup, steps)
            r["cusparse_ms"] = ms_c
            r["cusparse_over_ours"] = ms_c / ms
            del Acs
        except Exception as e:  # a reference point only: report why it is missing
            r["cusparse_unavailable"] = f"{type(e).__name__}: {e}"[:200]
        out[name] = r
        torch.cuda.empty_cache()

    c = W.laplacian_2d(512)
    one("laplacian2d_512", c.rows, c.cols, c.vals, c.m, c.n,
        "2D 5-point Laplacian 512^2 (n=262144, diag 4, off -1); working set < L2, flushed between calls")
    c = W.laplacian_3d(256)
    one("laplacian3d_256", c.rows, c.cols, c.vals, c.m, c.n, "3D 7-point Laplacian 256^3 (diag 6, off -1)")
    del c
    rows, cols, vals, n = W.rmat_device(22, 16, seed=1, device=dev)
    one("rmat22_f64", rows, cols, vals, n, n, "R-MAT scale 22 (0.57, 0.19, 0.19), edge factor 16, values N(0,1)")
    del rows, cols, vals
    torch.cuda.empty_cache()
    return out


def time_selector(dev, seeds=range(2000, 2050)):
    """Block-size selection on held-out matrices of the selector workload
    (seeds past the 2,000 training seeds; banded, block-diagonal, R-MAT, 2D /
    3D stencils, n log-uniform [10k, 4M]): the learned MLP's regret against
    the exhaustive min-bss sweep (block_statistics/consistency.cpp:147-173),
    next to every fixed block size, and the time of each way to choose."""
    import torch
    from abhsf_b200 import selector as sel
    from abhsf_b200 import workloads as W
    X, bits, pick = [], [], []
    t_learned = t_sweep = 0.0
    for seed in seeds:
        r, c, m, n, _ = W.selector_matrix(int(seed))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        f = sel.features(r, c, m, n)
        s = sel.predict(f)
        t1 = time.perf_counter()
        b, _ = sel.block_size_storage(r, c, m, n)
        t2 = time.perf_counter()
        t_learned += t1 - t0
        t_sweep += t2 - t1
        X.append(f)
        bits.append(b)
        pick.append(sel.SIZES.index(s))
        del r, c
    bits = np.array(bits)
    out = {"workload": f"{len(bits)} held-out selector matrices (seeds {seeds[0]}-{seeds[-1]})",
           "learned": sel.regret_summary(bits, np.array(pick)),
           "fixed": {str(s): sel.regret_summary(bits, np.full(len(bits), k)) for k, s in enumerate(sel.SIZES)},
           "learned_ms_per_matrix": 1e3 * t_learned / len(bits),
           "sweep_ms_per_matrix": 1e3 * t_sweep / len(bits)}
    out["choose_speedup"] = t_sweep / t_learned
    return out


def time_bstats(c, dev):
    """The reference's whole block-statistics sweep (the 64 block sizes 2..256 x
    2..256 of block_statistics/block_stats.cpp:144-170) on the timed matrix,
    inputs on the GPU: one abhsf_block_histogram call per size (one sort
    each, as the reference) against one abhsf_block_histogram_all call (one
    sort per column width)."""
    import torch
    from abhsf_b200 import block_histogram, block_histograms_all
    rows = torch.from_numpy(c.rows).to(dev)
    cols = torch.from_numpy(c.cols).to(dev)
    block_histograms_all(rows, cols, c.m, c.n)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    allh = block_histograms_all(rows, cols, c.m, c.n)
    t_all = time.perf_counter() - t0
    t0 = time.perf_counter()
    same = True
    for k in range(1, 9):
        for l in range(1, 9):
            h = block_histogram(rows, cols, c.m, c.n, 1 << k, 1 << l)
            same = same and h == allh[f"{1 << k}x{1 << l}"]
    t_per = time.perf_counter() - t0
    del rows, cols
    return {"workload": "the timed matrix, 64 block sizes", "per_size_s": t_per, "one_call_s": t_all,
            "speedup": t_per / t_all, "identical": same}


def cpu_reference_run(c, bytes_per_step: float, max_seconds: float, max_iters: int):
    """Reference CSR spmv_naive (oracle/_ref, compiled from the reference
    sources) on all host threads; falls back to the single-thread oracle port."""
    from oracle import oracle
    x = np.random.default_rng(X_SEED).uniform(-1, 1, c.n)
    y = np.zeros(c.m)
    if oracle.RefCSR.available():
        t0 = time.time()
        R = oracle.RefCSR(c.rows, c.cols, c.vals, c.m, c.n)
        log(f"reference CSR built in {time.time() - t0:.1f} s")
        for _ in range(4):  # warmup_iters, spmv/bottlenecks/spmv.cpp:33 (then up to its n_iters = 40)
            R.spmv(x, y)
        times = []
        t_start = time.perf_counter()
        while len(times) < max_iters and time.perf_counter() - t_start < max_seconds:
            t0 = time.perf_counter()
            R.spmv(x, y)
            times.append(time.perf_counter() - t0)
        cores = oracle.RefCSR.threads()
        R.release()
        kind = "reference"
        sample = (f"{len(times)} full y += A x of the same matrix, csr_matrix<double,int,int>::spmv_naive "
                  f"(spmv/bottlenecks/spmv.cpp:58-64) built from the reference sources, OpenMP static rows")
    else:
        oracle.spmv_elements(c.rows, c.cols, c.vals, x, y)
        times = []
        t_start = time.perf_counter()
        while len(times) < max_iters and time.perf_counter() - t_start < max_seconds:
            t0 = time.perf_counter()
            oracle.spmv_elements(c.rows, c.cols, c.vals, x, y)
            times.append(time.perf_counter() - t0)
        cores = 1
        kind = "port"
        sample = f"{len(times)} full y += A x with the oracle's element-order FP64 loop (1 thread)"
    t = sum(times) / len(times)  # the mean, as the GPU arm reports
    return {"value": bytes_per_step / t / 1e9, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample,
            "ms_per_step": t * 1e3, "gflops": 2.0 * c.nnz / t / 1e9}


def cpu_abhsf_run(c, bytes_per_step: float, max_seconds: float = 10.0, max_iters: int = 20):
    """A second CPU reference point: the project's C restatement of the ABHSF
    SpMV (the oracle's, the same format at s = 64) on all host threads
    (OpenMP over block rows), same matrix, same unit."""
    from oracle import oracle
    t0 = time.time()
    b = oracle.build(c.rows, c.cols, c.vals, c.m, c.n, 64)
    build_s = time.time() - t0
    x = np.random.default_rng(X_SEED).uniform(-1, 1, c.n)
    y = np.zeros(c.m)
    b.spmv_omp(x, y)  # warm-up
    times = []
    t_start = time.perf_counter()
    while len(times) < max_iters and time.perf_counter() - t_start < max_seconds:
        t1 = time.perf_counter()
        b.spmv_omp(x, y)
        times.append(time.perf_counter() - t1)
    t = statistics.median(times)
    cores = oracle.Built.threads()
    b.close()
    return {"value": bytes_per_step / t / 1e9, "unit": UNIT, "cores": cores, "kind": "port",
            "ms_per_step": t * 1e3, "build_s": build_s,
            "sample": f"{len(times)} full y += A x, the oracle's C ABHSF SpMV (s = 64) with OpenMP over block rows"}


def block_kernel_lines(text: str) -> list[dict]:
    """The result lines the reference's block micro-benchmarks print
    (spmv/orig/44_bitmap.cpp:759-768), colour codes removed."""
    text = re.sub(r"\x1b\[[0-9;]*m", "", text)
    lines = []
    for m in re.finditer(r"Block nonzeros =\s*(\d+), MFLOP/s: min =\s*([0-9.]+), avg =\s*([0-9.]+), "
                         r"max =\s*([0-9.]+); y-vector sum:\s*([0-9.eE+-]+)", text):
        lines.append({"bnnz": int(m.group(1)), "mflops_min": float(m.group(2)), "mflops_avg": float(m.group(3)),
                      "mflops_max": float(m.group(4)), "y_sum": float(m.group(5))})
    return lines


def cpu_block_kernel_run(max_seconds: float = 25.0):
    """The reference's format-level micro-baseline: its AVX2 4 x 4 bitmap
    block kernel spmv_temp (spmv/orig/44_bitmap.cpp:330-396), one thread, on
    its own synthetic matrix (8192 x 8192 identical random blocks, values 1,
    x = 1), compiled unmodified into oracle/_ref/44_bitmap.  It prints one
    line per block nonzero count, 1..16; the lines that arrive within
    max_seconds are kept (the run stops there)."""
    exe = os.path.join(ROOT, "oracle", "_ref", "44_bitmap")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/44_bitmap not built (make -C oracle ref)"}
    try:
        out = subprocess.run([exe, "4"], capture_output=True, timeout=max_seconds).stdout
    except subprocess.TimeoutExpired as e:
        out = e.stdout or b""
    lines = block_kernel_lines(out.decode(errors="replace"))
    return {"kernel": "44_bitmap spmv_temp (spmv/orig/44_bitmap.cpp:330-396), AVX2, 4 x 4 bitmap blocks",
            "unit": "MFLOP/s", "cores": 1, "kind": "reference", "lines": lines,
            "sample": f"the block nonzero counts finished within {max_seconds:.0f} s (of 1..16), "
                      "each 5 random patterns x 8 timed products over 8192^2 blocks"}


def ingest_run(c, max_entries: int = 3_000_000):
    """Matrix Market ingest, the path's data loader: the first max_entries
    elements of the workload written as a real general .mtx (17 significant
    digits), read by abhsf_read_mtx on all host threads and by the
    reference's read_mtx_real_or_binary (compiled from its sources into
    oracle/_ref/libref_mtx.so), best of two reads each, MB/s of file."""
    import ctypes as C
    import tempfile

    from abhsf_b200 import matrix as mx
    k = min(int(max_entries), c.nnz)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "sample.mtx")
        with open(p, "w") as f:
            f.write(f"%%MatrixMarket matrix coordinate real general\n{c.m} {c.n} {k}\n")
            step = 1 << 18
            for a in range(0, k, step):
                b = min(k, a + step)
                f.write("\n".join(f"{i} {j} {v:.17g}" for i, j, v in
                                  zip((c.rows[a:b] + 1).tolist(), (c.cols[a:b] + 1).tolist(), c.vals[a:b].tolist())))
                f.write("\n")
        size = os.path.getsize(p)
        ours = []
        for _ in range(2):
            t0 = time.perf_counter()
            got = mx.read_mtx(p)
            ours.append(time.perf_counter() - t0)
        out = {"entries": k, "file_bytes": size, "unit": "MB/s",
               "abhsf_read_mtx": {"MB/s": size / min(ours) / 1e6, "s": min(ours), "threads": os.cpu_count()}}
        try:  # the parse on the GPU: file read, copy, line scan, parse, checks, compaction
            import torch
            dev = []
            for _ in range(3):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                gd = mx.read_mtx_device(p)
                torch.cuda.synchronize()
                dev.append(time.perf_counter() - t0)
            same_d = (gd[0].numel() == got[0].size and np.array_equal(gd[0].cpu().numpy(), got[0])
                      and np.array_equal(gd[1].cpu().numpy(), got[1])
                      and np.array_equal(gd[2].cpu().numpy().view(np.uint64), got[2].view(np.uint64)))
            out["abhsf_read_mtx_device"] = {"MB/s": size / min(dev[1:]) / 1e6, "s": min(dev[1:]),
                                            "host_parsed": gd[5]["host_parsed"], "same_elements": bool(same_d)}
            del gd
        except Exception as exc:  # noqa: BLE001 -- reported, not fatal to the bench
            out["abhsf_read_mtx_device"] = {"error": str(exc)[:200]}
        lib = os.path.join(ROOT, "oracle", "_ref", "libref_mtx.so")
        if os.path.exists(lib):
            f_ = C.CDLL(lib).ref_mtx_read
            f_.restype = C.c_long
            rows = np.zeros(k, np.int64)
            cols = np.zeros(k, np.int64)
            vals = np.zeros(k)
            m_, n_ = C.c_long(), C.c_long()
            ref = []
            # the reference's reader logs to stdout, which carries only the JSON line
            sys.stdout.flush()
            saved = os.dup(1)
            null = os.open(os.devnull, os.O_WRONLY)
            try:
                os.dup2(null, 1)
                for _ in range(2):
                    t0 = time.perf_counter()
                    cnt = f_(os.fsencode(p), C.byref(m_), C.byref(n_), C.c_long(k), rows.ctypes.data_as(C.c_void_p),
                             cols.ctypes.data_as(C.c_void_p), vals.ctypes.data_as(C.c_void_p))
                    ref.append(time.perf_counter() - t0)
            finally:
                os.dup2(saved, 1)
                os.close(saved)
                os.close(null)
            same = (cnt == got[0].size and np.array_equal(rows[:cnt], got[0]) and np.array_equal(cols[:cnt], got[1])
                    and np.array_equal(vals[:cnt].view(np.uint64), got[2].view(np.uint64)))
            out["reference_reader"] = {"MB/s": size / min(ref) / 1e6, "s": min(ref), "threads": 1,
                                       "same_elements": bool(same)}
        else:
            out["reference_reader"] = {"unavailable": "oracle/_ref/libref_mtx.so not built"}
    return out


def build_format_stats(c):
    """Format statistics without a GPU (for the reference arm): the oracle
    builder gives the same bytes as the device format."""
    from oracle import oracle
    b = oracle.build(c.rows, c.cols, c.vals, c.m, c.n, 64)
    fmt = (b.M + 1) * 8 + b.T * 9 + (b.T + 1) * 16 + b.idx.size + b.values.size * 8
    return {"format_bytes": fmt}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    c = workload(args)
    st = build_format_stats(c)
    B = algorithmic_bytes(st, c.m, c.n)
    cpu = cpu_reference_run(c, B, max_seconds=30.0, max_iters=max(args.steps, 10))
    line = {
        "impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": cpu["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": c.name,
                   "nnz": c.nnz, "bytes_per_step": B, "gflops": cpu["gflops"]},
        "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist

    from abhsf_b200 import AbhsfMatrix

    from abhsf_b200.replicas import aggregate_rate, max_over_ranks, rank_info
    rank, local, world = rank_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)

    c = workload(args)
    t0 = time.time()
    A = AbhsfMatrix.from_elements(c.rows, c.cols, c.vals, c.m, c.n, block_size=64, sum_order=args.sum_order)
    torch.cuda.synchronize()
    build_s = time.time() - t0
    st = A.stats()
    B = algorithmic_bytes(st, c.m, c.n)
    log(f"built in {build_s:.2f} s: tiles {st['tiles']} {st['tiles_per_scheme']}, format {st['format_bytes']/1e6:.1f} MB, "
        f"B = {B/1e6:.1f} MB per step")

    rng = np.random.default_rng(X_SEED)
    x_h = rng.uniform(-1, 1, c.n)
    xd = torch.from_numpy(x_h).to(dev)
    yd = torch.zeros(c.m, dtype=torch.float64, device=dev)
    flush_w = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    flush_r = torch.ones(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)  # summed in place, no copy
    stream = torch.cuda.current_stream()

    def l2_flush():
        # write a buffer twice the L2, then read another: the read evicts the
        # written (dirty) lines, so their write-back happens here and not
        # inside the next timed SpMV, and L2 holds nothing of A, x or y
        flush_w.zero_()
        flush_r.sum()

    for _ in range(args.warmup):
        l2_flush()
        A.spmv(xd, yd)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    time.sleep(0.3)
    torch.cuda.synchronize()
    for k in range(args.steps):
        l2_flush()
        starts[k].record(stream)
        A.spmv(xd, yd)
        ends[k].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    times_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    t_mean = sum(times_ms) / len(times_ms)
    t_max = max_over_ranks(t_mean, dev)

    # e2e: host buffers (pinned), copies inside every step
    x_pin = torch.from_numpy(x_h).pin_memory().numpy()
    y_pin = torch.zeros(c.m, dtype=torch.float64).pin_memory().numpy()
    e2e_steps = 0 if args.no_e2e else args.steps
    for _ in range(max(2, args.warmup) if e2e_steps else 0):
        A.spmv(x_pin, y_pin)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        A.spmv(x_pin, y_pin)
    e2e_s = (time.perf_counter() - t0) / max(1, e2e_steps)
    e2e_s = max_over_ranks(e2e_s, dev)

    spmm = None if args.no_spmm else time_spmm(A, c, st, dev, stream, l2_flush, args.warmup)
    lowprec = None if args.no_lowprec else time_lowprec(c, dev, l2_flush, args.warmup)
    shapes = None if args.no_shapes or rank != 0 else time_shapes(dev, l2_flush, args.warmup)
    cg_times = None if args.no_cg or rank != 0 else time_cg(dev)
    batched = None if args.no_batched or rank != 0 else time_batched(dev, l2_flush, args.warmup)
    cusparse = None if args.no_cusparse or rank != 0 else time_cusparse(c, dev, l2_flush, args.warmup, t_mean)
    selector = None if args.no_selector or rank != 0 else time_selector(dev)
    bstats = None if args.no_bstats or rank != 0 else time_bstats(c, dev)

    peak, peak_src = hbm_peak()
    # every section's rate also as a fraction of the measured copy peak
    for sec in (spmm or {}).values():
        sec["frac_of_peak"] = sec["GB/s"] / peak
    for key in ("f32", "bf16"):
        if lowprec and key in lowprec:
            lowprec[key]["frac_of_peak"] = lowprec[key]["GB/s"] / peak
    if batched:
        for key in ("batched", "one_by_one"):
            batched[key]["frac_of_peak"] = batched[key]["GB/s"] / peak
    achieved = B / (t_mean * 1e-3) / 1e9
    cpu = cpu_abhsf = cpu_block = ingest = None
    status = A.device_status()
    if status:
        raise RuntimeError(f"SpMV kernel reported device status {status}")
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_run(c, B, max_seconds=20.0, max_iters=40)
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        try:
            cpu_abhsf = cpu_abhsf_run(c, B)
        except Exception as e:  # a secondary reference point: report why it is missing
            cpu_abhsf = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
        if not args.no_block_kernel:
            try:
                cpu_block = cpu_block_kernel_run()
            except Exception as e:
                cpu_block = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
        if not args.no_ingest:
            try:
                ingest = ingest_run(c)
            except Exception as e:
                ingest = {"unavailable": f"{type(e).__name__}: {e}"[:300]}
    if rank == 0:
        # every further measurement on a line of its own, the headline last
        sections = (("cpu_abhsf", cpu_abhsf), ("cpu_block_kernel", cpu_block), ("ingest", ingest),
                    ("block_stats_sweep", bstats), ("selector", selector), ("cusparse_csr", cusparse),
                    ("lowprec", lowprec), ("spmm", spmm), ("shapes", shapes), ("cg", cg_times),
                    ("batched", batched))
        for name, sec in sections:
            if sec is not None:
                print(json.dumps({"section": name, **sec}), flush=True)
        summary = {}
        if batched:
            summary["batched_ms"] = batched["batched"]["ms"]
            summary["batched_frac_of_peak"] = batched["batched"]["frac_of_peak"]
        if shapes:
            for k, v in shapes.items():
                summary[f"{k}_ms"] = v["ms"]
                if "cusparse_over_ours" in v:
                    summary[f"{k}_cusparse_over_ours"] = v["cusparse_over_ours"]
        if cg_times:
            summary["cg_plain_s"] = cg_times["plain"]["seconds"]
            summary["cg_tuned_bf16_s"] = cg_times["tuned_bf16"]["seconds"]
            summary["cg_tuned_bf16_speedup"] = cg_times["tuned_bf16_speedup"]
        if spmm:
            summary["spmm_frac_of_peak"] = {k: v["frac_of_peak"] for k, v in spmm.items()}
        if cusparse and "ours_speedup" in cusparse:
            summary["cusparse_over_ours"] = cusparse["ours_speedup"]
        line = {
            "metric": METRIC, "value": aggregate_rate(B, t_max * 1e-3, world), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {
                "workload": c.name,
                "block_size": 64, "nnz": c.nnz, "tiles": st["tiles"], "tiles_per_scheme": st["tiles_per_scheme"],
                "bytes_per_step": B, "format_bytes": st["format_bytes"], "spmv_bytes": st["spmv_bytes"],
                "msmf_min_bytes_per_step": st["msmf_bits"][6] // 8 + 8 * c.n + 16 * c.m,
                "csr_bytes_per_step": 12 * c.nnz + 4 * (c.m + 1) + 8 * c.n + 16 * c.m,
                "l2": "between steps a 256 MiB buffer is written, then another 256 MiB read (dirty lines written back before the timed SpMV); working set 600 MB > 126 MB L2",
                "gflops": 2.0 * c.nnz / (t_mean * 1e-3) / 1e9, "build_s": build_s,
                "parallelism": f"replicas x{world}", "sum_order": args.sum_order,
                "kernels_per_step": A.kernels(),
            },
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": ncu_traffic_per_launch(args.sum_order, c.n) if args.matrix == "tiled_mixture" else None,
                         "peak_source": peak_src,
                         "kernel": KERNELS[args.sum_order] + "<64>"},
            "cpu_baseline": cpu,
            "e2e": None if not e2e_steps else {
                "value": aggregate_rate(B, e2e_s, world), "unit": UNIT, "h2d_bytes_per_step": 8 * c.n + 8 * c.m,
                "d2h_bytes_per_step": 8 * c.m, "ms_per_step": e2e_s * 1e3},
            "summary": summary,
            "gpu_launches": args.steps * A.kernels(),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    A.release()
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ingest", action="store_true",
                    help="skip the Matrix Market ingest timing (ours against the reference's reader, 3M entries)")
    ap.add_argument("--no-block-kernel", action="store_true",
                    help="skip the reference's 4 x 4 bitmap block micro-baseline (25 s on one host core)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer loop (profiling runs)")
    ap.add_argument("--no-spmm", action="store_true", help="skip the multi-right-hand-side timings")
    ap.add_argument("--no-lowprec", action="store_true", help="skip the f32 / bf16 SpMV timings")
    ap.add_argument("--no-cg", action="store_true", help="skip the CG solves on the 3D Laplacian")
    ap.add_argument("--no-shapes", action="store_true",
                    help="skip the 2D / 3D Laplacian and R-MAT scale 22 SpMVs (with cuSPARSE beside them)")
    ap.add_argument("--no-batched", action="store_true", help="skip the 256-matrix batched launch")
    ap.add_argument("--no-cusparse", action="store_true", help="skip the cuSPARSE CSR reference point")
    ap.add_argument("--no-selector", action="store_true", help="skip the block-size selector evaluation")
    ap.add_argument("--no-bstats", action="store_true", help="skip the 64-size block-statistics sweep")
    ap.add_argument("--sum-order", choices=["reference", "tree"], default="reference",
                    help="reference: bitwise the reference CSR's y; tree: warp reduction trees")
    ap.add_argument("--n", type=int, default=DEFAULT_N,
                    help="matrix order of the tiled mixture (smaller only for profiling captures)")
    ap.add_argument("--matrix", choices=["tiled_mixture", "laplacian3d", "rmat22"], default="tiled_mixture",
                    help="the timed matrix (laplacian3d and rmat22 for profiling those cases)")
    ap.add_argument("--grid", type=int, default=128, help="grid side of --matrix laplacian3d")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
