"""ctypes wrapper of the CPU oracle (oracle/abhsf_oracle.c) and of the
reference's own CSR SpMV built into oracle/_ref (oracle/ref_csr_harness.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, always as the checker or the timed
CPU baseline, never as the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_CSR_PATH = os.path.join(REF_DIR, "libref_csr.so")

COO, CSR, BITMAP, DENSE = 0, 1, 2, 3
TYPE_BINARY, TYPE_INTEGER, TYPE_REAL, TYPE_COMPLEX = 0, 1, 2, 3
VAL_F64, VAL_F32, VAL_BF16 = 0, 1, 2
VALUE_TYPES = {"f64": VAL_F64, "f32": VAL_F32, "bf16": VAL_BF16}
ERRORS = {1: "invalid argument", 2: "index out of range", 3: "duplicate entry",
          4: "out of memory", 5: "unsupported"}

_i64p = C.POINTER(C.c_int64)
_u64p = C.POINTER(C.c_uint64)
_f64p = C.POINTER(C.c_double)


class OrcMatrix(C.Structure):
    _fields_ = [
        ("m", C.c_int64), ("n", C.c_int64), ("nnz", C.c_int64),
        ("s", C.c_int32), ("log2s", C.c_int32),
        ("M", C.c_int64), ("N", C.c_int64), ("T", C.c_int64),
        ("value_type", C.c_int32),
        ("n_values", C.c_int64), ("idx_bytes", C.c_int64),
        ("brow_ptr", _i64p), ("tile_col", C.POINTER(C.c_uint32)),
        ("tile_nnz", C.POINTER(C.c_uint32)), ("tile_scheme", C.POINTER(C.c_uint8)),
        ("tile_val_off", _i64p), ("tile_idx_off", _i64p),
        ("idx", C.POINTER(C.c_uint8)), ("values", C.c_void_p),
    ]


def build_lib() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "liborc.so"], check=True)


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_lib()
        L = C.CDLL(LIB_PATH)
        u64 = C.c_uint64
        for name, nargs in (("orc_block_coo_bits", 3), ("orc_block_csr_bits", 3)):
            getattr(L, name).restype = u64
            getattr(L, name).argtypes = [u64] * nargs
        L.orc_ceil_log2.restype = u64
        L.orc_ceil_log2.argtypes = [u64]
        L.orc_block_bitmap_bits.restype = u64
        L.orc_block_bitmap_bits.argtypes = [u64, u64]
        L.orc_block_dense_bits.restype = u64
        L.orc_block_dense_bits.argtypes = [u64, u64, u64, u64]
        for name in ("orc_block_min_bits", "orc_block_min_bits_wocsr"):
            getattr(L, name).restype = u64
            getattr(L, name).argtypes = [u64, u64, u64, u64, C.c_int]
        L.orc_select_scheme.restype = C.c_int
        L.orc_select_scheme.argtypes = [u64, u64, u64, u64, C.c_int, C.c_int]
        L.orc_block_histogram.restype = C.c_int64
        L.orc_block_histogram.argtypes = [_i64p, _i64p, C.c_int64, C.c_int, C.c_int, _u64p]
        L.orc_mmf_line.restype = None
        L.orc_mmf_line.argtypes = [u64, u64, u64, C.c_int, u64, u64, _u64p, u64, _u64p, _u64p]
        L.orc_build.restype = C.c_int
        L.orc_build.argtypes = [_i64p, _i64p, _f64p, C.c_int64, C.c_int64, C.c_int64, C.c_int32,
                                C.c_int32, u64, C.c_int32, C.c_int32, C.c_int32,
                                C.POINTER(C.POINTER(OrcMatrix))]
        L.orc_free.restype = None
        L.orc_free.argtypes = [C.POINTER(OrcMatrix)]
        L.orc_spmv_abhsf.restype = None
        L.orc_spmv_abhsf.argtypes = [C.POINTER(OrcMatrix), _f64p, _f64p]
        L.orc_spmv_abhsf_omp.restype = None
        L.orc_spmv_abhsf_omp.argtypes = [C.POINTER(OrcMatrix), _f64p, _f64p]
        L.orc_omp_threads.restype = C.c_int
        L.orc_omp_threads.argtypes = []
        for name in ("orc_spmv_elements", "orc_abs_spmv_elements"):
            getattr(L, name).restype = None
            getattr(L, name).argtypes = [_i64p, _i64p, _f64p, C.c_int64, _f64p, _f64p]
        f32p = C.POINTER(C.c_float)
        L.orc_spmv_elements_f32.restype = None
        L.orc_spmv_elements_f32.argtypes = [_i64p, _i64p, f32p, C.c_int64, f32p, f32p]
        L.orc_values_as_f32.restype = None
        L.orc_values_as_f32.argtypes = [_f64p, C.c_int64, C.c_int, f32p]
        L.orc_slices_build.restype = C.c_int
        L.orc_slices_build.argtypes = [C.POINTER(OrcMatrix), C.c_double, C.POINTER(C.POINTER(OrcSlices))]
        L.orc_slices_free.restype = None
        L.orc_slices_free.argtypes = [C.POINTER(OrcSlices)]
        L.orc_spmv_slices.restype = None
        L.orc_spmv_slices.argtypes = [C.POINTER(OrcMatrix), C.POINTER(OrcSlices), _f64p, _f64p]
        _lib = L
    return _lib


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)


# ----------------------------------------------------------------- cost model
def ceil_log2(v: int) -> int:
    return int(lib().orc_ceil_log2(v))


def block_bits(scheme: int, r: int, s: int, nnz: int, bits: int = 64) -> int:
    L = lib()
    if scheme == COO:
        return int(L.orc_block_coo_bits(r, s, nnz))
    if scheme == CSR:
        return int(L.orc_block_csr_bits(r, s, nnz))
    if scheme == BITMAP:
        return int(L.orc_block_bitmap_bits(r, s))
    return int(L.orc_block_dense_bits(r, s, nnz, bits))


def block_min_bits(r, s, nnz, bits, is_binary=False, allow_csr=True) -> int:
    f = lib().orc_block_min_bits if allow_csr else lib().orc_block_min_bits_wocsr
    return int(f(r, s, nnz, bits, int(is_binary)))


def select_scheme(r, s, nnz, bits, is_binary=False, allow_csr=True) -> int:
    return int(lib().orc_select_scheme(r, s, nnz, bits, int(is_binary), int(allow_csr)))


# ----------------------------------------------------------------- stats
def block_histogram(rows, cols, k: int, l: int) -> dict[int, int]:
    """block nnz -> number of blocks for block size 2^k x 2^l."""
    rows, cols = _i64(rows), _i64(cols)
    hist = np.zeros((1 << k) * (1 << l) + 1, dtype=np.uint64)
    rc = lib().orc_block_histogram(_p(rows, _i64p), _p(cols, _i64p), rows.size, k, l, _p(hist, _u64p))
    if rc < 0:
        raise RuntimeError("oracle histogram: " + ERRORS.get(-rc, str(rc)))
    nz = np.nonzero(hist)[0]
    return {int(z): int(hist[z]) for z in nz}


def mmf_line(m, n, nnz, mtype, r, s, hist: dict[int, int]):
    """(single[8], double[8]) = coo32 csr32 coo csr bitmap dense abhsf abhsf134."""
    zmax = max(hist) if hist else 0
    h = np.zeros(zmax + 1, dtype=np.uint64)
    for z, c in hist.items():
        h[z] = c
    o1 = np.zeros(8, dtype=np.uint64)
    o2 = np.zeros(8, dtype=np.uint64)
    lib().orc_mmf_line(m, n, nnz, mtype, r, s, _p(h, _u64p), h.size, _p(o1, _u64p), _p(o2, _u64p))
    return [int(v) for v in o1], [int(v) for v in o2]


# ----------------------------------------------------------------- builder
class OrcSlices(C.Structure):
    _fields_ = [("n", C.c_int64), ("slots", C.c_int64), ("lane_records", C.c_int64), ("E", C.c_int64),
                ("block_rows", C.c_int64), ("base", C.POINTER(C.c_int64)), ("meta", C.POINTER(C.c_int64)),
                ("brow", C.POINTER(C.c_uint32)), ("steps", C.POINTER(C.c_uint32)), ("lanes", C.POINTER(C.c_uint32)),
                ("chain", C.POINTER(C.c_uint8)), ("lane", C.POINTER(C.c_uint32)), ("words", C.POINTER(C.c_uint32)),
                ("vidx", C.POINTER(C.c_int64))]


class Built:
    """Host copy of the arrays the oracle builder emits."""

    def __init__(self, ptr):
        self._ptr = ptr
        a = ptr.contents
        self.m, self.n, self.nnz, self.s = a.m, a.n, a.nnz, a.s
        self.M, self.N, self.T = a.M, a.N, a.T
        self.value_type = a.value_type
        T = a.T

        def arr(p, count, dt):
            if count == 0:
                return np.zeros(0, dtype=dt)
            return np.ctypeslib.as_array(p, shape=(count,)).astype(dt, copy=True)

        self.brow_ptr = arr(a.brow_ptr, a.M + 1, np.int64)
        self.tile_col = arr(a.tile_col, T, np.uint32)
        self.tile_nnz = arr(a.tile_nnz, T, np.uint32)
        self.tile_scheme = arr(a.tile_scheme, T, np.uint8)
        self.tile_val_off = arr(a.tile_val_off, T + 1, np.int64)
        self.tile_idx_off = arr(a.tile_idx_off, T + 1, np.int64)
        self.idx = arr(a.idx, a.idx_bytes, np.uint8)
        vdt = {VAL_F64: np.float64, VAL_F32: np.float32, VAL_BF16: np.uint16}[a.value_type]
        if a.n_values:
            buf = (C.c_uint8 * (a.n_values * np.dtype(vdt).itemsize)).from_address(a.values)
            self.values = np.frombuffer(buf, dtype=vdt).copy()
        else:
            self.values = np.zeros(0, dtype=vdt)

    def spmv(self, x: np.ndarray, y: np.ndarray) -> None:
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert y.dtype == np.float64 and y.flags.c_contiguous
        lib().orc_spmv_abhsf(self._ptr, _p(x, _f64p), _p(y, _f64p))

    def spmv_omp(self, x: np.ndarray, y: np.ndarray) -> None:
        """y += A x on all host threads (bitwise spmv's y)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert y.dtype == np.float64 and y.flags.c_contiguous
        lib().orc_spmv_abhsf_omp(self._ptr, _p(x, _f64p), _p(y, _f64p))

    @staticmethod
    def threads() -> int:
        return int(lib().orc_omp_threads())

    def slices(self, avg: float) -> dict:
        """The delta-coded row slices of the hypersparse block rows
        (orc_slices_build): per-slice arrays in slice order, the lane
        records, and every slot's word and value index (-1: padding)."""
        out = C.POINTER(OrcSlices)()
        rc = lib().orc_slices_build(self._ptr, float(avg), C.byref(out))
        try:
            if rc != 0:
                raise ValueError("oracle slices: " + ERRORS.get(rc, str(rc)))
            P = out.contents

            def arr(ptr, count, dt):
                if count == 0:
                    return np.zeros(0, dtype=dt)
                return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)

            res = {"slices": int(P.n), "slots": int(P.slots), "lane_records": int(P.lane_records),
                   "elements": int(P.E), "block_rows": int(P.block_rows)}
            for k, dt in (("base", np.int64), ("meta", np.int64), ("brow", np.uint32), ("steps", np.uint32),
                          ("lanes", np.uint32), ("chain", np.uint8)):
                res[k] = arr(getattr(P, k), P.n, dt)
            res["lane"] = arr(P.lane, P.lane_records, np.uint32)
            res["words"] = arr(P.words, P.slots, np.uint32)
            res["vidx"] = arr(P.vidx, P.slots, np.int64)
            return res
        finally:
            lib().orc_slices_free(out)

    def spmv_slices(self, avg: float, x: np.ndarray, y: np.ndarray) -> None:
        """y += A x over the slice rows only, decoding the oracle's slices."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert y.dtype == np.float64 and y.flags.c_contiguous
        out = C.POINTER(OrcSlices)()
        rc = lib().orc_slices_build(self._ptr, float(avg), C.byref(out))
        try:
            if rc != 0:
                raise ValueError("oracle slices: " + ERRORS.get(rc, str(rc)))
            lib().orc_spmv_slices(self._ptr, out, _p(x, _f64p), _p(y, _f64p))
        finally:
            lib().orc_slices_free(out)

    def close(self):
        if self._ptr is not None:
            lib().orc_free(self._ptr)
            self._ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build(rows, cols, vals, m, n, s, value_type="f64", bits=64, is_binary=False,
          allow_csr=True, forced_scheme=-1) -> Built:
    rows, cols = _i64(rows), _i64(cols)
    vals = None if vals is None else np.ascontiguousarray(vals, dtype=np.float64)
    out = C.POINTER(OrcMatrix)()
    rc = lib().orc_build(_p(rows, _i64p), _p(cols, _i64p),
                         None if vals is None else _p(vals, _f64p), rows.size, m, n, s,
                         VALUE_TYPES[value_type], bits, int(is_binary), int(allow_csr),
                         int(forced_scheme), C.byref(out))
    if rc != 0:
        raise ValueError("oracle build: " + ERRORS.get(rc, str(rc)))
    return Built(out)


# ----------------------------------------------------------------- SpMV
def spmv_elements(rows, cols, vals, x, y=None) -> np.ndarray:
    """y += A x in element order (spmv/unified/spmv.cpp:1195-1201)."""
    rows, cols = _i64(rows), _i64(cols)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    if y is None:
        y = np.zeros(int(rows.max()) + 1 if rows.size else 0, dtype=np.float64)
    lib().orc_spmv_elements(_p(rows, _i64p), _p(cols, _i64p), _p(vals, _f64p), rows.size,
                            _p(x, _f64p), _p(y, _f64p))
    return y


def values_as_f32(vals, value_type: str) -> np.ndarray:
    """Values as a matrix stored as `value_type` ("f32" / "bf16") holds them,
    widened to f32 (orc_values_as_f32)."""
    v = np.ascontiguousarray(vals, dtype=np.float64)
    out = np.empty(v.size, dtype=np.float32)
    lib().orc_values_as_f32(_p(v, _f64p), v.size, VALUE_TYPES[value_type], _p(out, C.POINTER(C.c_float)))
    return out


def spmv_elements_f32(rows, cols, vals_f32, x_f32, y_f32) -> np.ndarray:
    """The element-order loop in f32 (orc_spmv_elements_f32)."""
    rows, cols = _i64(rows), _i64(cols)
    vals = np.ascontiguousarray(vals_f32, dtype=np.float32)
    x = np.ascontiguousarray(x_f32, dtype=np.float32)
    y = np.array(y_f32, dtype=np.float32, copy=True)
    f32p = C.POINTER(C.c_float)
    lib().orc_spmv_elements_f32(_p(rows, _i64p), _p(cols, _i64p), _p(vals, f32p), rows.size, _p(x, f32p), _p(y, f32p))
    return y


def abs_spmv(rows, cols, vals, x, m) -> np.ndarray:
    rows, cols = _i64(rows), _i64(cols)
    vals = np.ascontiguousarray(vals, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(m, dtype=np.float64)
    lib().orc_abs_spmv_elements(_p(rows, _i64p), _p(cols, _i64p), _p(vals, _f64p), rows.size,
                                _p(x, _f64p), _p(out, _f64p))
    return out


# ----------------------------------------------------------------- reference CSR
class RefCSR:
    """The reference's csr_matrix<double,int,int> with spmv_naive, compiled from
    the reference sources into oracle/_ref/libref_csr.so."""

    _L = None

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(REF_CSR_PATH)

    @classmethod
    def _lib(cls):
        if cls._L is None:
            L = C.CDLL(REF_CSR_PATH)
            L.ref_csr_create.restype = C.c_void_p
            L.ref_csr_create.argtypes = [_i64p, _i64p, _f64p, C.c_long, C.c_long, C.c_long]
            L.ref_csr_spmv_naive.restype = None
            L.ref_csr_spmv_naive.argtypes = [C.c_void_p, _f64p, _f64p]
            L.ref_csr_release.restype = None
            L.ref_csr_release.argtypes = [C.c_void_p]
            L.ref_csr_max_threads.restype = C.c_int
            cls._L = L
        return cls._L

    def __init__(self, rows, cols, vals, m, n):
        rows, cols = _i64(rows), _i64(cols)
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        self.m, self.n = m, n
        self._h = self._lib().ref_csr_create(_p(rows, _i64p), _p(cols, _i64p), _p(vals, _f64p),
                                             rows.size, m, n)

    def spmv(self, x: np.ndarray, y: np.ndarray) -> None:
        assert x.dtype == np.float64 and y.dtype == np.float64
        self._lib().ref_csr_spmv_naive(self._h, _p(x, _f64p), _p(y, _f64p))

    @classmethod
    def threads(cls) -> int:
        return int(cls._lib().ref_csr_max_threads())

    def release(self):
        if self._h:
            self._lib().ref_csr_release(self._h)
            self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
