"""Block-size selection: the exhaustive min-bss sweep and the learned MLP.

The reference picks the block size of a matrix by computing its block
statistics at every candidate size and taking the one of least storage
(block_statistics/min-bss.cpp:14-58), and scores restricted choices by their
regret, the storage above the minimum in percent, averaged and maximised over
matrices (block_statistics/consistency.cpp:140-174).

Here the sweep runs on the GPU (abhsf_block_size_storage: five block
histograms, sizes 16..256) and a small MLP (12 features -> 64 -> 64 -> 5,
ReLU, FP32; abhsf_selector_features / abhsf_mlp_*) predicts its answer from
one pass of features.  The network is trained on the GPU by the library's own
forward, backward and Adam kernels; this module holds the data set, the
training loop and the regret report:

    python -m abhsf_b200.selector train --out DIR [--train 2000 --heldout 200]

writes DIR/selector_model.inc (the model built into the library, copied to
abhsf_b200/csrc/), DIR/selector_model.f32, DIR/selector_data.npz (features
and storage of every matrix), DIR/selector_heldout.npz (the held-out part,
copied to tests/golden/) and DIR/selector_report.json.

The same network trained on measured time instead of storage:

    python -m abhsf_b200.selector train-time --out DIR [--train 1500 --heldout 300] [--data DIR/selector_time_data.npz]

labels each matrix with the FP64 SpMV time at each size (median of five
launches of the default build), targets softmax(-excess time / tau), picks
tau and the number of steps on a validation fifth of the training matrices,
and writes DIR/selector_model_time.inc (copied to abhsf_b200/csrc/, the model
of ABHSF_SELECT_LEARNED_TIME), DIR/selector_time_data.npz (every matrix's
features, storage and times; --data reuses it instead of timing anew),
DIR/selector_time_heldout.npz (copied to tests/golden/) and
DIR/selector_time_report.json (regret in time and in storage of the model,
of the storage model, of min-bss and of every fixed size).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import time

import numpy as np

from . import capi

F, H, NC, P = capi.FEATURES, capi.MLP_HIDDEN, capi.MLP_CLASSES, capi.MLP_PARAMS
SIZES = capi.BLOCK_SIZES
# parameter offsets, the layout of include/abhsf/abhsf_gpu.h
OW1 = 0
OB1 = OW1 + F * H
OW2 = OB1 + H
OB2 = OW2 + H * H
OW3 = OB2 + H
OB3 = OW3 + H * NC
OMEAN = OB3 + NC
OISTD = OMEAN + F
TRAINABLE = OMEAN


# ---------------------------------------------------------------- library calls

def _stream_ptr(stream=None):
    import torch
    if not torch.cuda.is_available():
        return None
    return (stream or torch.cuda.current_stream()).cuda_stream


def _coo_args(rows, cols):
    import torch
    on_dev = isinstance(rows, torch.Tensor) and rows.is_cuda
    if on_dev:
        rows = rows.to(torch.int64).contiguous()
        cols = cols.to(torch.int64).contiguous()
        return rows, cols, rows.numel(), rows.data_ptr(), cols.data_ptr(), True
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int64)
    return rows, cols, rows.size, rows.ctypes.data, cols.ctypes.data, False


def block_size_storage(rows, cols, m: int, n: int, allow_csr: bool = True, value_type: str = "f64",
                       stream=None) -> tuple[np.ndarray, int]:
    """ABHSF storage in bits at block sizes 16..256 (uint64[5]) and the size
    of least storage (ties to the smaller)."""
    rows, cols, nnz, rp, cp, on_dev = _coo_args(rows, cols)
    o = capi.BuildOpts()
    capi.lib.abhsf_build_opts_default(C.byref(o))
    o.inputs_on_device = int(on_dev)
    o.allow_csr = int(allow_csr)
    o.value_type = capi.VALUE_TYPES[value_type]
    bits = np.zeros(5, np.uint64)
    best = C.c_int32()
    capi.check(capi.lib.abhsf_block_size_storage(rp if nnz else None, cp if nnz else None, nnz, int(m), int(n),
                                                 C.byref(o), _stream_ptr(stream),
                                                 bits.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(best)))
    return bits, int(best.value)


MMF_COLUMNS = ("coo32", "csr32", "coo", "csr", "bitmap", "dense", "abhsf", "abhsf134")


def mmf_table(hists: dict, m: int, n: int, nnz: int, matrix_type: str = "real") -> dict:
    """The 64 lines of the reference's mmf-single and mmf-double
    (block_statistics/mmf.cpp:53-138) from the 64 block histograms
    (matrix.block_histograms_all, one GPU call): {(h, w): (single[8],
    double[8])}, columns MMF_COLUMNS, bits with values included."""
    from .matrix import mmf_line
    out = {}
    for key, h in hists.items():
        r, s = (int(t) for t in key.split("x"))
        out[(r, s)] = tuple(mmf_line(m, n, nnz, matrix_type, r, s, h))
    return out


def min_bss(table: dict, precision: str = "double") -> dict:
    """One matrix's column of the reference's mmf-bss-single / -double
    (block_statistics/min-bss.cpp:35-55): per block size (h, w), ascending,
    the least storage over the coo, csr, bitmap, dense and abhsf columns."""
    i = {"single": 0, "double": 1}[precision]
    return {bs: min(lines[i][2:7]) for bs, lines in sorted(table.items())}


def block_opt(table: dict, precision: str = "double") -> tuple[tuple[int, int], str, int]:
    """mmf_t::block_opt (block_statistics/mmf.h:77-102): the least storage
    over every block size and the coo .. abhsf columns, visited in the
    reference's order (block sizes ascending by (h, w), then the columns),
    the first strict minimum kept.  Returns ((h, w), column, bits)."""
    i = {"single": 0, "double": 1}[precision]
    best = None
    for bs, lines in sorted(table.items()):
        for k in range(2, 7):
            v = lines[i][k]
            if best is None or v < best[2]:
                best = (bs, MMF_COLUMNS[k], v)
    if best is None:
        raise ValueError("empty table")
    return best


def min_schemes(table: dict, precision: str = "double") -> tuple[list[int], tuple[int, int]]:
    """One matrix's line of the reference's mmf-schemes-single / -double
    (block_statistics/min-schemes.cpp:24-44): each of the eight mmf columns'
    least storage over all 64 block sizes, and block_opt's block size."""
    i = {"single": 0, "double": 1}[precision]
    mins = [min(r[i][k] for r in table.values()) for k in range(8)]
    return mins, block_opt(table, precision)[0]


def _size_sets() -> dict[str, list[tuple[int, int]]]:
    """The restricted block-size sets of block_statistics/consistency.cpp:101-123."""
    b8 = [(h, h) for h in (2, 4, 8, 16, 32, 64, 128, 256)]
    b14 = sorted(set(b8) | {(h, w) for h in (4, 8, 16) for w in (4, 8, 16)})
    b20 = sorted(set(b8) | {(h, w) for h in (4, 8, 16, 32) for w in (4, 8, 16, 32)})
    b64 = [(h, w) for h in (2, 4, 8, 16, 32, 64, 128, 256) for w in (2, 4, 8, 16, 32, 64, 128, 256)]
    return {"B_64": b64, "B_20": b20, "B_14": b14, "B_8": b8}


def consistency(tables: list[dict], scheme: str = "adaptive", precision: str = "double") -> dict:
    """The reference's consistency study (block_statistics/consistency.cpp:
    56-188) over matrices' mmf tables: per matrix the least storage over all
    64 sizes and the coo, csr, bitmap, dense and abhsf columns; the storage
    at a block size is abhsf134 ("adaptive") or the least of coo, bitmap and
    dense plus 2 tag bits ("min-fixed"), both without CSR; for each of the
    size sets B_64, B_20, B_14 and B_8 the excess of the set's best size
    over that least storage, in percent: {set: (average, maximum)}."""
    i = {"single": 0, "double": 1}[precision]
    if scheme not in ("adaptive", "min-fixed"):
        raise ValueError("scheme: adaptive or min-fixed")
    if not tables:
        raise ValueError("no matrices")
    sets = _size_sets()
    acc = {k: [] for k in sets}
    for t in tables:
        least = min(min(min(r[i][2:6]), r[i][6]) for r in t.values())
        at = {}
        for bs, r in t.items():
            coo, csr, bitmap, dense, abhsf, abhsf134 = r[i][2:8]
            at[bs] = min(coo, bitmap, dense) + 2 if scheme == "min-fixed" else abhsf134
        for k, members in sets.items():
            acc[k].append((min(at[bs] for bs in members) - least) / least * 100.0)
    return {k: (float(np.mean(v)), float(np.max(v))) for k, v in acc.items()}


def features(rows, cols, m: int, n: int, stream=None) -> np.ndarray:
    """The selector's 12 features of a matrix (float32), computed on the GPU."""
    rows, cols, nnz, rp, cp, on_dev = _coo_args(rows, cols)
    out = np.zeros(F, np.float32)
    capi.check(capi.lib.abhsf_selector_features(rp if nnz else None, cp if nnz else None, nnz, int(m), int(n),
                                                int(on_dev), _stream_ptr(stream),
                                                out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def builtin_model() -> np.ndarray:
    """The model built into the library (float32[MLP_PARAMS]), trained on storage."""
    out = np.zeros(P, np.float32)
    capi.check(capi.lib.abhsf_selector_builtin_model(out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def builtin_time_model() -> np.ndarray:
    """The model built into the library that was trained on measured SpMV time."""
    out = np.zeros(P, np.float32)
    capi.check(capi.lib.abhsf_selector_builtin_time_model(out.ctypes.data_as(C.POINTER(C.c_float))))
    return out


def predict(feats: np.ndarray, model: np.ndarray | None = None, stream=None) -> int:
    """Block size the model (None = built-in) predicts for one feature vector."""
    feats = np.ascontiguousarray(feats, dtype=np.float32)
    mp = None if model is None else np.ascontiguousarray(model, dtype=np.float32)
    bs = C.c_int32()
    capi.check(capi.lib.abhsf_selector_predict(None if mp is None else mp.ctypes.data,
                                               feats.ctypes.data_as(C.POINTER(C.c_float)), _stream_ptr(stream),
                                               C.byref(bs)))
    return int(bs.value)


def autotune(rows, cols, vals, m: int, n: int, candidates=SIZES, reps: int = 10, value_type: str = "f64",
             keep: bool = False, stream=None):
    """Block size by measured SpMV time (abhsf_autotune): the matrix is built
    at each candidate size and reps SpMVs of it are timed on the stream.
    Returns (ms per SpMV at sizes 16..256, -1 where not timed; the fastest
    size; that size's AbhsfMatrix when keep, else None)."""
    from .matrix import AbhsfMatrix
    rows, cols, nnz, rp, cp, on_dev = _coo_args(rows, cols)
    if vals is not None:
        if on_dev:
            import torch
            vals = vals.to(torch.float64).contiguous()
            vp = vals.data_ptr()
        else:
            vals = np.ascontiguousarray(vals, dtype=np.float64)
            vp = vals.ctypes.data
    o = capi.BuildOpts()
    capi.lib.abhsf_build_opts_default(C.byref(o))
    o.inputs_on_device = int(on_dev)
    o.value_type = capi.VALUE_TYPES[value_type]
    mask = sum(1 << SIZES.index(s) for s in candidates)
    ms = np.zeros(5, np.float32)
    best = C.c_int32()
    h = C.c_void_p()
    capi.check(capi.lib.abhsf_autotune(rp if nnz else None, cp if nnz else None,
                                       vp if (vals is not None and nnz) else None, nnz, int(m), int(n), C.byref(o),
                                       mask, int(reps), _stream_ptr(stream),
                                       ms.ctypes.data_as(C.POINTER(C.c_float)), C.byref(best),
                                       C.byref(h) if keep else None))
    A = None
    if keep:
        A = AbhsfMatrix()
        A._h = h
        A.m, A.n, A.nnz = int(m), int(n), int(nnz)
        A.block_size = int(best.value)
        A.value_type = value_type
    return ms, int(best.value), A


class Mlp:
    """The selector network on the GPU: parameters, Adam moments and the
    library's forward / backward / Adam kernels over torch buffers."""

    def __init__(self, params: np.ndarray):
        import torch
        self.p = torch.from_numpy(np.ascontiguousarray(params, dtype=np.float32)).cuda()
        self.m = torch.zeros(P, dtype=torch.float32, device="cuda")
        self.v = torch.zeros(P, dtype=torch.float32, device="cuda")
        self.g = torch.zeros(P, dtype=torch.float32, device="cuda")
        self.loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        self.step_count = 0

    def forward(self, x, keep: bool = False):
        """probs[batch][5] (and the activations when keep) for x[batch][12] (CUDA float32)."""
        import torch
        b = x.shape[0]
        probs = torch.empty(b, NC, dtype=torch.float32, device="cuda")
        act = torch.empty(b, 2 * H, dtype=torch.float32, device="cuda") if keep else None
        capi.check(capi.lib.abhsf_mlp_forward(self.p.data_ptr(), x.data_ptr(), b, probs.data_ptr(),
                                              act.data_ptr() if keep else None, _stream_ptr()))
        return (probs, act) if keep else probs

    def backward(self, x, targets, probs, act):
        """Fills self.g (trainable part) and self.loss."""
        import torch
        b = x.shape[0]
        delta = torch.empty(b, NC + 2 * H, dtype=torch.float32, device="cuda")
        capi.check(capi.lib.abhsf_mlp_backward(self.p.data_ptr(), x.data_ptr(), targets.data_ptr(), b,
                                               probs.data_ptr(), act.data_ptr(), delta.data_ptr(),
                                               self.g.data_ptr(), self.loss.data_ptr(), _stream_ptr()))

    def adam(self, lr: float):
        self.step_count += 1
        capi.check(capi.lib.abhsf_mlp_adam(self.p.data_ptr(), self.g.data_ptr(), self.m.data_ptr(),
                                           self.v.data_ptr(), self.step_count, float(lr), _stream_ptr()))

    def params(self) -> np.ndarray:
        return self.p.cpu().numpy().copy()


# ---------------------------------------------------------------- host logic

def init_params(x_train: np.ndarray, seed: int = 0) -> np.ndarray:
    """He-initialised weights, zero biases, and the input normalisation
    (mean, 1 / stdev) of the training features."""
    rng = np.random.default_rng(seed)
    p = np.zeros(P, np.float32)
    p[OW1:OB1] = rng.standard_normal(F * H) * np.sqrt(2.0 / F)
    p[OW2:OB2] = rng.standard_normal(H * H) * np.sqrt(2.0 / H)
    p[OW3:OB3] = rng.standard_normal(H * NC) * np.sqrt(2.0 / H)
    mean = x_train.mean(axis=0)
    std = x_train.std(axis=0)
    p[OMEAN:OISTD] = mean
    p[OISTD:OISTD + F] = np.where(std > 1e-6, 1.0 / np.maximum(std, 1e-6), 1.0)
    return p


def targets_from_bits(bits: np.ndarray, tau: float = 0.0) -> np.ndarray:
    """Training targets from the storage of each size: the one-hot argmin
    (tau = 0) or a softmax of -excess / tau over the sizes, excess being the
    storage above the minimum as a fraction of it."""
    b = bits.astype(np.float64)
    mn = b.min(axis=1, keepdims=True)
    if tau <= 0:
        t = np.zeros_like(b)
        t[np.arange(b.shape[0]), b.argmin(axis=1)] = 1.0
        return t.astype(np.float32)
    z = -(b - mn) / mn / tau
    z -= z.max(axis=1, keepdims=True)
    e = np.exp(z)
    return (e / e.sum(axis=1, keepdims=True)).astype(np.float32)


def targets_from_times(ms: np.ndarray, tau: float = 0.05) -> np.ndarray:
    """Training targets from the measured SpMV time at each size: a softmax of
    -excess / tau, excess being the time above the fastest as a fraction of it
    (sizes without a time, ms <= 0, get no weight)."""
    t = np.where(ms > 0, ms.astype(np.float64), np.inf)
    mn = t.min(axis=1, keepdims=True)
    z = -(t - mn) / mn / tau
    z -= z.max(axis=1, keepdims=True)
    e = np.exp(z)
    return (e / e.sum(axis=1, keepdims=True)).astype(np.float32)


def time_regret_summary(ms: np.ndarray, choice: np.ndarray) -> dict:
    """Per matrix the SpMV time at the chosen size over the fastest one, minus
    one, in percent (the storage regret of consistency.cpp:147-160 with time
    in place of storage): its average and maximum, the share of matrices whose
    choice is the fastest, and the summed time of the choices over the summed
    fastest times."""
    t = np.where(ms > 0, ms.astype(np.float64), np.inf)
    mn = t.min(axis=1)
    got = t[np.arange(t.shape[0]), choice]
    r = (got - mn) / mn * 100.0
    return {"avg_pct": float(r.mean()), "max_pct": float(r.max()), "exact": float((r == 0).mean()),
            "total_over_best": float(got.sum() / mn.sum())}


def regret(bits: np.ndarray, choice: np.ndarray) -> np.ndarray:
    """Per matrix: (storage of the chosen size - least storage) / least
    storage * 100 (block_statistics/consistency.cpp:147-160); choice holds
    indices 0..4 into bits' columns."""
    b = bits.astype(np.float64)
    mn = b.min(axis=1)
    return (b[np.arange(b.shape[0]), choice] - mn) / mn * 100.0


def regret_summary(bits: np.ndarray, choice: np.ndarray) -> dict:
    """Average and maximum regret over matrices (consistency.cpp:161-173),
    and the share of matrices whose choice is a minimum."""
    r = regret(bits, choice)
    return {"avg_pct": float(r.mean()), "max_pct": float(r.max()), "exact": float((r == 0).mean())}


def write_model_inc(params: np.ndarray, path: str, name: str = "kBuiltinModel",
                    what: str = "Trained block-size selector") -> None:
    """The model as the C++ initialiser selector.cu includes."""
    params = np.asarray(params, dtype=np.float32)
    assert params.size == P
    lines = [f"// {what}: ABHSF_MLP_PARAMS floats in the layout of",
             "// include/abhsf/abhsf_gpu.h.  Written by abhsf_b200/selector.py; do not edit.",
             f"static const float {name}[ABHSF_MLP_PARAMS] = {{"]
    vals = [np.format_float_scientific(v, precision=8, unique=False) + "f" for v in params]
    for i in range(0, P, 8):
        lines.append("    " + ", ".join(vals[i:i + 8]) + ",")
    lines.append("};")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def untrained_model() -> np.ndarray:
    """A model that always predicts block size 64 (zero weights, b3 one-hot)."""
    p = np.zeros(P, np.float32)
    p[OB3 + SIZES.index(64)] = 1.0
    p[OISTD:OISTD + F] = 1.0
    return p


# ---------------------------------------------------------------- data and training

def dataset(seeds, n_min=10_000, n_max=4_000_000, nnz_max=16_000_000, log=None):
    """Features (float32[len][12]) and storage at sizes 16..256
    (uint64[len][5]) of the selector workload's matrices, both on the GPU."""
    import torch
    from . import workloads as W
    X = np.zeros((len(seeds), F), np.float32)
    B = np.zeros((len(seeds), 5), np.uint64)
    names = []
    t_feat = t_sweep = 0.0
    for i, seed in enumerate(seeds):
        rows, cols, m, n, name = W.selector_matrix(int(seed), n_min, n_max, nnz_max)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        X[i] = features(rows, cols, m, n)
        t1 = time.perf_counter()
        B[i], _ = block_size_storage(rows, cols, m, n)
        t2 = time.perf_counter()
        t_feat += t1 - t0
        t_sweep += t2 - t1
        names.append(name)
        if log and (i + 1) % 200 == 0:
            log(f"{i + 1}/{len(seeds)} matrices  features {t_feat:.1f}s  sweep {t_sweep:.1f}s")
        del rows, cols
    return X, B, names, {"features_s": t_feat, "sweep_s": t_sweep}


def train(X: np.ndarray, bits: np.ndarray, steps: int = 6000, batch: int = 256, lr: float = 3e-3,
          tau: float = 0.02, seed: int = 0, log=None, targets: np.ndarray | None = None) -> np.ndarray:
    """Adam on the GPU kernels, mini-batches drawn by numpy's default_rng(seed),
    learning rate decayed by cosine to lr / 20.  Targets: from the storage
    (targets_from_bits(bits, tau)) unless given."""
    import torch
    net = Mlp(init_params(X, seed))
    xt = torch.from_numpy(X).cuda()
    tt = torch.from_numpy(targets_from_bits(bits, tau) if targets is None else targets).cuda()
    rng = np.random.default_rng(seed)
    for step in range(steps):
        idx = torch.from_numpy(rng.integers(0, X.shape[0], min(batch, X.shape[0]))).cuda()
        xb, tb = xt[idx].contiguous(), tt[idx].contiguous()
        probs, act = net.forward(xb, keep=True)
        net.backward(xb, tb, probs, act)
        net.adam(lr * (0.05 + 0.95 * 0.5 * (1 + np.cos(np.pi * step / steps))))
        if log and (step + 1) % 1000 == 0:
            log(f"step {step + 1}  loss {float(net.loss):.4f}")
    return net.params()


def time_dataset(seeds, n_min=10_000, n_max=2_000_000, nnz_max=8_000_000, reps=5, log=None):
    """Features, storage at sizes 16..256 and the measured FP64 SpMV time at
    each size (ms, the median of reps CUDA-event-timed launches after two;
    the library's default build at that size, values N(0,1)) of the selector
    workload's matrices."""
    import torch
    from . import workloads as W
    from .matrix import AbhsfMatrix
    X = np.zeros((len(seeds), F), np.float32)
    B = np.zeros((len(seeds), 5), np.uint64)
    T = np.zeros((len(seeds), 5), np.float32)
    names = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for i, seed in enumerate(seeds):
        rows, cols, m, n, name = W.selector_matrix(int(seed), n_min, n_max, nnz_max)
        g = torch.Generator(device=rows.device)
        g.manual_seed(int(seed))
        vals = torch.randn(rows.numel(), dtype=torch.float64, device=rows.device, generator=g)
        X[i] = features(rows, cols, m, n)
        B[i], _ = block_size_storage(rows, cols, m, n)
        x = torch.rand(n, dtype=torch.float64, device=rows.device)
        y = torch.zeros(m, dtype=torch.float64, device=rows.device)
        for k, s in enumerate(SIZES):
            A = AbhsfMatrix.from_elements(rows, cols, vals, m, n, block_size=s)
            for _ in range(2):
                A.spmv(x, y)
            ts = []
            for _ in range(reps):
                e0.record()
                A.spmv(x, y)
                e1.record()
                e1.synchronize()
                ts.append(e0.elapsed_time(e1))
            T[i, k] = float(np.median(ts))
            A.release()
        names.append(name)
        if log and (i + 1) % 50 == 0:
            log(f"{i + 1}/{len(seeds)} matrices timed")
        del rows, cols, vals, x, y
    return X, B, T, names


def choose(model: np.ndarray, X: np.ndarray) -> np.ndarray:
    """Indices 0..4 of the sizes the model picks for each row of X, through
    the library's forward kernel."""
    import torch
    net = Mlp(model)
    probs = net.forward(torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda())
    return probs.argmax(dim=1).cpu().numpy()


def main_time(args) -> int:
    """train-time: the selector trained on measured SpMV times.  The targets'
    temperature and the number of steps are picked on a validation split (the
    last fifth of the training matrices), the model then trained on all of
    them; the held-out matrices are only scored."""
    os.makedirs(args.out, exist_ok=True)

    def log(msg):
        print(msg, flush=True)

    if args.data:
        d = np.load(args.data)
        Xtr, Btr, Ttr = d["X_train"], d["bits_train"], d["ms_train"]
        Xho, Bho, Tho, nho = d["X_heldout"], d["bits_heldout"], d["ms_heldout"], list(d["names_heldout"])
    else:
        seeds_train = np.arange(args.train)
        seeds_held = np.arange(2000, 2000 + args.heldout)
        Xtr, Btr, Ttr, ntr = time_dataset(seeds_train, n_max=args.n_max, log=log)
        Xho, Bho, Tho, nho = time_dataset(seeds_held, n_max=args.n_max, log=log)
        np.savez_compressed(os.path.join(args.out, "selector_time_data.npz"), X_train=Xtr, bits_train=Btr,
                            ms_train=Ttr, names_train=np.array(ntr), X_heldout=Xho, bits_heldout=Bho, ms_heldout=Tho,
                            names_heldout=np.array(nho))
    np.savez_compressed(os.path.join(args.out, "selector_time_heldout.npz"), X=Xho, bits=Bho, ms=Tho,
                        names=np.array(nho))
    cut = (4 * Xtr.shape[0]) // 5
    search = {}
    for tau in (0.05, 0.15, 0.4):
        for steps in (500, 1500, 4000):
            mdl = train(Xtr[:cut], Btr[:cut], steps=steps, targets=targets_from_times(Ttr[:cut], tau))
            search[f"tau={tau} steps={steps}"] = time_regret_summary(Ttr[cut:], choose(mdl, Xtr[cut:]))
    best = min(search, key=lambda k: (search[k]["total_over_best"], search[k]["avg_pct"]))
    tau, steps = (float(v.split("=")[1]) for v in best.split())
    log(f"validation: {json.dumps(search)}\nchosen: {best}")
    t0 = time.perf_counter()
    model = train(Xtr, Btr, steps=int(steps), log=log, targets=targets_from_times(Ttr, tau))
    t_train = time.perf_counter() - t0
    model.tofile(os.path.join(args.out, "selector_model_time.f32"))
    write_model_inc(model, os.path.join(args.out, "selector_model_time.inc"), "kBuiltinTimeModel",
                    "Block-size selector trained on measured SpMV times")
    report = {"train": int(Xtr.shape[0]), "heldout": int(Xho.shape[0]), "train_s": t_train, "chosen": best,
              "validation": search}
    for split, X, B, T in (("train", Xtr, Btr, Ttr), ("heldout", Xho, Bho, Tho)):
        c_time = choose(model, X)
        c_store = choose(builtin_model(), X)
        minbss = B.astype(np.float64).argmin(axis=1)
        report[split + "_time_model"] = {"time": time_regret_summary(T, c_time), "storage": regret_summary(B, c_time)}
        report[split + "_storage_model"] = {"time": time_regret_summary(T, c_store),
                                            "storage": regret_summary(B, c_store)}
        report[split + "_minbss"] = {"time": time_regret_summary(T, minbss), "storage": regret_summary(B, minbss)}
        for s in SIZES:
            k = np.full(B.shape[0], SIZES.index(s))
            report[f"{split}_fixed{s}"] = {"time": time_regret_summary(T, k), "storage": regret_summary(B, k)}
    with open(os.path.join(args.out, "selector_time_report.json"), "w") as f:
        json.dump(report, f, indent=1)
    log(json.dumps(report))
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("cmd", choices=["train", "train-time"])
    ap.add_argument("--out", required=True)
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--heldout", type=int, default=200)
    ap.add_argument("--n-max", type=int, default=4_000_000)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--data", help="train-time: a saved selector_time_data.npz instead of timing anew")
    args = ap.parse_args(argv)
    if args.cmd == "train-time":
        return main_time(args)
    os.makedirs(args.out, exist_ok=True)

    def log(msg):
        print(msg, flush=True)

    seeds_train = np.arange(args.train)
    seeds_held = np.arange(args.train, args.train + args.heldout)
    Xtr, Btr, ntr, ttr = dataset(seeds_train, n_max=args.n_max, log=log)
    Xho, Bho, nho, tho = dataset(seeds_held, n_max=args.n_max, log=log)
    np.savez_compressed(os.path.join(args.out, "selector_data.npz"), X_train=Xtr, bits_train=Btr,
                        X_heldout=Xho, bits_heldout=Bho, names_train=np.array(ntr), names_heldout=np.array(nho))
    # the held-out part alone: the fixture tests/golden/selector_heldout.npz
    np.savez_compressed(os.path.join(args.out, "selector_heldout.npz"), X=Xho, bits=Bho, names=np.array(nho))
    t0 = time.perf_counter()
    model = train(Xtr, Btr, steps=args.steps, log=log)
    t_train = time.perf_counter() - t0
    model.tofile(os.path.join(args.out, "selector_model.f32"))
    write_model_inc(model, os.path.join(args.out, "selector_model.inc"))
    report = {"train": len(seeds_train), "heldout": len(seeds_held), "train_s": t_train,
              "features_s_heldout": tho["features_s"], "sweep_s_heldout": tho["sweep_s"]}
    for split, X, B in (("train", Xtr, Btr), ("heldout", Xho, Bho)):
        report[split + "_learned"] = regret_summary(B, choose(model, X))
        for s in SIZES:
            report[f"{split}_fixed{s}"] = regret_summary(B, np.full(B.shape[0], SIZES.index(s)))
        report[split + "_label_counts"] = np.bincount(B.astype(np.float64).argmin(axis=1), minlength=5).tolist()
    with open(os.path.join(args.out, "selector_report.json"), "w") as f:
        json.dump(report, f, indent=1)
    log(json.dumps(report))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
