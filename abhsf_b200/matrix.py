"""Host-side mirror of the reference's per-format matrix class.

The reference's formats share one shape (spmv/unified/spmv.cpp:74-127,
140-159, 210-226; spmv/bottlenecks/spmv.cpp:43-64,125-133):

    A.from_elements(elements, props)   # build
    A.spmv(x, y)                       # y += A x
    A.release()                        # free

:class:`AbhsfMatrix` keeps that shape over the C ABI of libabhsf_b200.so.
Inputs are numpy arrays (host memory) or torch CUDA tensors (device memory);
``spmv`` on CUDA tensors is ordered on torch's current stream, on numpy
arrays it copies through the device and returns when y holds the result.
Errors raise :class:`abhsf_b200.capi.AbhsfError` subclasses, the analogue of
the reference's ``std::runtime_error``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import capi

try:  # torch is plumbing only: device memory and streams
    import torch
except ImportError:  # pragma: no cover
    torch = None


def _is_cuda(t) -> bool:
    return torch is not None and isinstance(t, torch.Tensor) and t.is_cuda


def _stream_ptr(stream=None) -> int | None:
    if stream is not None:
        return int(stream.cuda_stream) if hasattr(stream, "cuda_stream") else int(stream)
    if torch is not None and torch.cuda.is_available():
        return int(torch.cuda.current_stream().cuda_stream)
    return None


def _ptr(a) -> int:
    if _is_cuda(a):
        return a.data_ptr()
    return a.ctypes.data


def _opts(block_size, value_type, allow_csr, matrix_type, forced_scheme, bits_per_value, on_device,
          sum_order="reference", selector="minbss", selector_model=None, slice_tile_nnz=0) -> capi.BuildOpts:
    o = capi.BuildOpts()
    capi.lib.abhsf_build_opts_default(C.byref(o))
    o.block_size = 0 if block_size == "auto" else int(block_size)
    o.selector = capi.SELECTORS[selector]
    if selector_model is not None:
        if selector_model.dtype != np.float32 or selector_model.size != capi.MLP_PARAMS \
                or not selector_model.flags.c_contiguous:
            raise capi.InvalidValue(capi.INVALID_VALUE, f"selector_model must be {capi.MLP_PARAMS} contiguous float32")
        o.selector_model = selector_model.ctypes.data
    o.value_type = capi.VALUE_TYPES[value_type]
    o.allow_csr = 1 if allow_csr else 0
    o.matrix_type = capi.MATRIX_TYPES[matrix_type]
    if forced_scheme is None:
        o.forced_scheme = -1
    else:
        o.forced_scheme = capi.SCHEME_NAMES.index(forced_scheme) if isinstance(forced_scheme, str) else int(forced_scheme)
    o.bits_per_value = int(bits_per_value)
    o.inputs_on_device = 1 if on_device else 0
    o.sum_order = capi.SUM_ORDERS[sum_order]
    o.slice_tile_nnz = int(slice_tile_nnz)
    return o


class AbhsfMatrix:
    """ABHSF matrix resident on the GPU."""

    def __init__(self):
        self._h = None
        self.m = self.n = self.nnz = 0
        self.block_size = 0
        self.value_type = "f64"

    # ------------------------------------------------------------------ build
    @classmethod
    def from_elements(cls, rows, cols, vals, m: int, n: int, *, block_size: int | str = 64,
                      value_type: str = "f64", allow_csr: bool = True, matrix_type: str = "real",
                      forced_scheme=None, bits_per_value: int = 0, sum_order: str = "reference",
                      selector: str = "minbss", selector_model=None, slice_tile_nnz: int = 0,
                      stream=None) -> "AbhsfMatrix":
        """Builds from COO triplets (0-based, any order, no duplicates).
        Scheme per tile by exact minimum storage (msmf.h:35-63) unless
        forced_scheme names one.  vals may be None for binary matrices.
        sum_order "reference" makes spmv bitwise equal to the reference's CSR
        spmv_naive; "tree" uses warp reduction trees.  block_size "auto"
        lets `selector` choose it: "minbss" (least storage over 16..256, the
        exhaustive sweep) or "learned" (the MLP; selector_model: float32
        parameters, None = the built-in model).  slice_tile_nnz: block rows
        whose tiles hold at most this many elements on average are summed
        from delta-coded row slices (0: the library's default, -1: none)."""
        on_dev = _is_cuda(rows)
        if on_dev:
            if not (_is_cuda(cols) and (vals is None or _is_cuda(vals))):
                raise capi.InvalidValue(capi.INVALID_VALUE, "rows, cols and vals must all be host or all be CUDA")
            rows = rows.to(torch.int64).contiguous()
            cols = cols.to(torch.int64).contiguous()
            vals = None if vals is None else vals.to(torch.float64).contiguous()
        else:
            rows = np.ascontiguousarray(rows, dtype=np.int64)
            cols = np.ascontiguousarray(cols, dtype=np.int64)
            vals = None if vals is None else np.ascontiguousarray(vals, dtype=np.float64)
        nnz = int(rows.numel() if on_dev else rows.size)
        if (cols.numel() if on_dev else cols.size) != nnz or (
                vals is not None and (vals.numel() if on_dev else vals.size) != nnz):
            raise capi.InvalidValue(capi.INVALID_VALUE, "rows, cols and vals differ in length")
        o = _opts(block_size, value_type, allow_csr, matrix_type, forced_scheme, bits_per_value, on_dev, sum_order,
                  selector, selector_model, slice_tile_nnz)
        h = C.c_void_p()
        capi.check(capi.lib.abhsf_build(_ptr(rows) if nnz else None, _ptr(cols) if nnz else None,
                                        _ptr(vals) if (vals is not None and nnz) else None, nnz, int(m), int(n),
                                        C.byref(o), _stream_ptr(stream), C.byref(h)))
        A = cls()
        A._h = h
        A.m, A.n, A.nnz = int(m), int(n), nnz
        A.value_type = value_type
        A.block_size = A.stats()["block_size"] if block_size == "auto" else int(block_size)
        return A

    # ------------------------------------------------------------------ spmv
    def spmv(self, x, y, stream=None) -> None:
        """y += A x.  CUDA tensors: asynchronous on the (current) stream;
        numpy arrays: synchronous through device staging buffers."""
        self._check_open()
        if _is_cuda(x) or _is_cuda(y):
            if not (_is_cuda(x) and _is_cuda(y)):
                raise capi.InvalidValue(capi.INVALID_VALUE, "x and y must both be CUDA tensors or both numpy")
            self._check_vec(x, y, torch.float64, x.numel(), y.numel(), x.is_contiguous() and y.is_contiguous())
            capi.check(capi.lib.abhsf_spmv(self._h, x.data_ptr(), y.data_ptr(), _stream_ptr(stream)))
        else:
            if not (isinstance(x, np.ndarray) and isinstance(y, np.ndarray)):
                raise capi.InvalidValue(capi.INVALID_VALUE, "x and y must be numpy arrays or CUDA tensors")
            self._check_vec(x, y, np.float64, x.size, y.size, x.flags.c_contiguous and y.flags.c_contiguous)
            capi.check(capi.lib.abhsf_spmv_host(self._h, x.ctypes.data, y.ctypes.data, _stream_ptr(stream)))

    def spmv_f32(self, x, y, stream=None) -> None:
        """y += A x in f32 (matrix stored as f32 or bf16); CUDA float32
        tensors, asynchronous on the stream."""
        self._check_open()
        if not (_is_cuda(x) and _is_cuda(y)):
            raise capi.InvalidValue(capi.INVALID_VALUE, "x and y must be CUDA tensors")
        self._check_vec(x, y, torch.float32, x.numel(), y.numel(), x.is_contiguous() and y.is_contiguous())
        capi.check(capi.lib.abhsf_spmv_f32(self._h, x.data_ptr(), y.data_ptr(), _stream_ptr(stream)))

    def spmm(self, X, Y, stream=None) -> None:
        """Y += A X for 2-D CUDA float64 tensors X (n x k) and Y (m x k) whose
        rows are contiguous (stride 1 along k), asynchronous on the stream."""
        self._check_open()
        if not (_is_cuda(X) and _is_cuda(Y)):
            raise capi.InvalidValue(capi.INVALID_VALUE, "X and Y must be CUDA tensors")
        if X.dim() != 2 or Y.dim() != 2 or X.shape[0] != self.n or Y.shape[0] != self.m or X.shape[1] != Y.shape[1]:
            raise capi.InvalidValue(capi.INVALID_VALUE, f"X must be {self.n} x k and Y {self.m} x k")
        if X.dtype != torch.float64 or Y.dtype != torch.float64:
            raise capi.InvalidValue(capi.INVALID_VALUE, "X and Y must be float64")
        k = X.shape[1]
        if k and ((X.stride(1) != 1 and X.shape[0] > 0) or (Y.stride(1) != 1 and Y.shape[0] > 0)):
            raise capi.InvalidValue(capi.INVALID_VALUE, "X and Y rows must be contiguous")
        ldx, ldy = max(X.stride(0), k), max(Y.stride(0), k)
        capi.check(capi.lib.abhsf_spmm(self._h, k, X.data_ptr(), ldx, Y.data_ptr(), ldy, _stream_ptr(stream)))

    def _check_vec(self, x, y, dtype, nx, ny, contiguous):
        if x.dtype != dtype or y.dtype != dtype:
            raise capi.InvalidValue(capi.INVALID_VALUE, f"x and y must be {dtype}, got {x.dtype}, {y.dtype}")
        if nx != self.n or ny != self.m:
            raise capi.InvalidValue(capi.INVALID_VALUE, f"x must have n={self.n} and y m={self.m} entries")
        if not contiguous:
            raise capi.InvalidValue(capi.INVALID_VALUE, "x and y must be contiguous")

    # ------------------------------------------------------------------ release
    def release(self) -> None:
        if self._h is not None and self._h.value:
            capi.check(capi.lib.abhsf_release(self._h))
        self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.release()

    def _check_open(self):
        if self._h is None or not self._h.value:
            raise capi.InvalidValue(capi.INVALID_VALUE, "matrix was released or never built")

    @property
    def handle(self) -> int:
        self._check_open()
        return int(self._h.value)

    def device_status(self, clear: bool = False, stream=None) -> int:
        """ABHSF_DEVSTAT_* bits raised by kernels on this matrix (0 = none);
        waits for the stream."""
        self._check_open()
        v = C.c_int32()
        capi.check(capi.lib.abhsf_device_status(self._h, _stream_ptr(stream), int(clear), C.byref(v)))
        return int(v.value)

    # ------------------------------------------------------------------ introspection
    def stats(self) -> dict:
        self._check_open()
        s = capi.Stats()
        capi.check(capi.lib.abhsf_stats_get(self._h, C.byref(s)))
        return {
            "m": s.m, "n": s.n, "nnz": s.nnz, "block_size": s.block_size,
            "value_type": [k for k, v in capi.VALUE_TYPES.items() if v == s.value_type][0],
            "block_rows": s.block_rows, "block_cols": s.block_cols, "tiles": s.tiles,
            "tiles_per_scheme": dict(zip(capi.SCHEME_NAMES, list(s.tiles_per_scheme))),
            "nnz_per_scheme": dict(zip(capi.SCHEME_NAMES, list(s.nnz_per_scheme))),
            "stored_values": s.stored_values, "payload_bytes": s.payload_bytes, "format_bytes": s.format_bytes,
            "msmf_bits": list(s.msmf_bits), "spmv_bytes": s.spmv_bytes,
        }

    def export(self) -> dict:
        """Host copies of every format array (layout in include/abhsf/abhsf_gpu.h)."""
        st = self.stats()
        T, M = st["tiles"], st["block_rows"]
        vdt = {"f64": np.float64, "f32": np.float32, "bf16": np.uint16}[st["value_type"]]
        out = {
            "brow_ptr": np.zeros(M + 1, np.int64), "tile_col": np.zeros(T, np.uint32),
            "tile_nnz": np.zeros(T, np.uint32), "tile_scheme": np.zeros(T, np.uint8),
            "tile_val_off": np.zeros(T + 1, np.int64), "tile_idx_off": np.zeros(T + 1, np.int64),
            "payload": np.zeros(st["payload_bytes"], np.uint8), "values": np.zeros(st["stored_values"], vdt),
        }
        p = [out[k].ctypes.data if out[k].size else None for k in
             ("brow_ptr", "tile_col", "tile_nnz", "tile_scheme", "tile_val_off", "tile_idx_off", "payload", "values")]
        capi.check(capi.lib.abhsf_export_host(self._h, *p))
        return out

    def kernels(self) -> int:
        """Kernels one spmv of this matrix launches (abhsf_spmv_kernels)."""
        self._check_open()
        v = C.c_int32()
        capi.check(capi.lib.abhsf_spmv_kernels(self._h, C.byref(v)))
        return int(v.value)

    def slices(self) -> dict:
        """The delta-coded row slices the SpMV reads for the hypersparse block
        rows (abhsf_slices_info / abhsf_slices_export): per-slice arrays in
        slice order, the lane records, and the words and values of every slot."""
        self._check_open()
        ns, nslot, nlr, ne, nb = (C.c_int64() for _ in range(5))
        capi.check(capi.lib.abhsf_slices_info(self._h, C.byref(ns), C.byref(nslot), C.byref(nlr), C.byref(ne),
                                              C.byref(nb)))
        S, SL, LR = ns.value, nslot.value, nlr.value
        vdt = {"f64": np.float64, "f32": np.float32, "bf16": np.uint16}[self.value_type]
        out = {"slices": S, "slots": SL, "lane_records": LR, "elements": ne.value, "block_rows": nb.value,
               "base": np.zeros(S, np.int64), "meta": np.zeros(S, np.int64), "brow": np.zeros(S, np.uint32),
               "steps": np.zeros(S, np.uint32), "lanes": np.zeros(S, np.uint32), "chain": np.zeros(S, np.uint8),
               "lane": np.zeros(LR, np.uint32), "words": np.zeros(SL, np.uint32), "values": np.zeros(SL, vdt)}
        keys = ("base", "meta", "brow", "steps", "lanes", "chain", "lane", "words", "values")
        capi.check(capi.lib.abhsf_slices_export(self._h, *[out[k].ctypes.data if out[k].size else None
                                                          for k in keys]))
        return out


# ---------------------------------------------------------------------- block statistics
def block_histogram(rows, cols, m: int, n: int, r: int, s: int, stream=None) -> dict[int, int]:
    """block nnz -> number of r x s blocks, computed on the GPU
    (block_statistics/block_stats.cpp:69-100)."""
    on_dev = _is_cuda(rows)
    if on_dev:
        rows = rows.to(torch.int64).contiguous()
        cols = cols.to(torch.int64).contiguous()
        nnz = rows.numel()
    else:
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        cols = np.ascontiguousarray(cols, dtype=np.int64)
        nnz = rows.size
    hist = np.zeros(r * s + 1, dtype=np.uint64)
    blocks = C.c_int64()
    capi.check(capi.lib.abhsf_block_histogram(_ptr(rows) if nnz else None, _ptr(cols) if nnz else None, nnz, m, n,
                                              r, s, 1 if on_dev else 0, _stream_ptr(stream),
                                              hist.ctypes.data_as(capi._u64p), hist.size, C.byref(blocks)))
    nz = np.nonzero(hist)[0]
    return {int(z): int(hist[z]) for z in nz}


def block_histograms_all(rows, cols, m: int, n: int, stream=None) -> dict[str, dict[int, int]]:
    """"RxS" -> {block nnz: blocks} for all 64 block sizes 2..256 x 2..256 in one
    GPU call (the 64 .bstats files of block_statistics/block_stats.cpp:144-170)."""
    on_dev = _is_cuda(rows)
    if on_dev:
        rows = rows.to(torch.int64).contiguous()
        cols = cols.to(torch.int64).contiguous()
        nnz = rows.numel()
    else:
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        cols = np.ascontiguousarray(cols, dtype=np.int64)
        nnz = rows.size
    hist = np.zeros(capi.BSTATS_ALL_LEN, dtype=np.uint64)
    blocks = np.zeros(64, dtype=np.int64)
    capi.check(capi.lib.abhsf_block_histogram_all(_ptr(rows) if nnz else None, _ptr(cols) if nnz else None, nnz, m, n,
                                                  1 if on_dev else 0, _stream_ptr(stream),
                                                  hist.ctypes.data_as(capi._u64p),
                                                  blocks.ctypes.data_as(C.POINTER(C.c_int64))))
    out, off = {}, 0
    for p in range(64):
        r, s = 2 << (p // 8), 2 << (p % 8)
        h = hist[off:off + r * s + 1]
        nz = np.nonzero(h)[0]
        out[f"{r}x{s}"] = {int(z): int(h[z]) for z in nz}
        assert sum(out[f"{r}x{s}"].values()) == blocks[p]
        off += r * s + 1
    return out


def _coo_result(c: "capi.CooHost"):
    """(rows, cols, vals, m, n, info) copied out of a library-owned CooHost,
    which is freed."""
    try:
        k = int(c.nnz)
        rows = np.ctypeslib.as_array(c.rows, shape=(k,)).copy() if k else np.zeros(0, np.int64)
        cols = np.ctypeslib.as_array(c.cols, shape=(k,)).copy() if k else np.zeros(0, np.int64)
        vals = np.ctypeslib.as_array(c.vals, shape=(k,)).copy() if k else np.zeros(0, np.float64)
        info = {"matrix_type": {0: "binary", 2: "real"}[int(c.matrix_type)],
                "symmetry": _SYMMETRIES[int(c.symmetry)],
                "stored_triangle": ("", "lower", "upper")[int(c.stored_triangle)]}
        return rows, cols, vals, int(c.m), int(c.n), info
    finally:
        capi.lib.abhsf_coo_host_free(C.byref(c))


_SYMMETRIES = ("symmetric", "hermitian", "skew", "general")


def read_mtx(path: str, threads: int = 0):
    """A Matrix Market coordinate file as the reference's read_mtx_real_or_binary
    reads it (include/abhsf/utils/matrix_market_reader.h:146-200), parsed on
    the host by the library: (rows, cols, vals, m, n, info) with 0-based int64
    indices, float64 values, info = {"matrix_type", "symmetry",
    "stored_triangle"}."""
    c = capi.CooHost()
    capi.check(capi.lib.abhsf_read_mtx(os.fsencode(path), int(threads), C.byref(c)))
    return _coo_result(c)


def read_mtx_device(path: str, stream=None):
    """read_mtx with the entry lines parsed on the GPU (abhsf_read_mtx_device):
    (rows, cols, vals, m, n, info) as CUDA tensors (int64, int64, float64),
    the elements read_mtx returns, in the same order; info also says how many
    entries the host parsed ("host_parsed": spellings the device leaves to
    it)."""
    c = capi.CooDevice()
    capi.check(capi.lib.abhsf_read_mtx_device(os.fsencode(path), _stream_ptr(stream), C.byref(c)))
    try:
        k = int(c.nnz)
        rows = torch.empty(k, dtype=torch.int64, device="cuda")
        cols = torch.empty(k, dtype=torch.int64, device="cuda")
        vals = torch.empty(k, dtype=torch.float64, device="cuda")
        if k:
            capi.check(capi.lib.abhsf_coo_device_copy(C.byref(c), rows.data_ptr(), cols.data_ptr(), vals.data_ptr(),
                                                       _stream_ptr(stream)))
            torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
        info = {"matrix_type": {0: "binary", 2: "real"}[int(c.matrix_type)],
                "symmetry": _SYMMETRIES[int(c.symmetry)],
                "stored_triangle": ("", "lower", "upper")[int(c.stored_triangle)],
                "host_parsed": int(c.host_parsed)}
        return rows, cols, vals, int(c.m), int(c.n), info
    finally:
        capi.lib.abhsf_coo_device_free(C.byref(c))


def expand_symmetric(rows, cols, vals, symmetry: str):
    """The whole matrix from the stored triangle of a symmetric, skew or
    hermitian (real) file, as read_mtx returns it: every off-diagonal element
    (i, j, v) gains its mirror (j, i, v), or (j, i, -v) for skew, the
    pairs block_statistics/block_stats.cpp:122-127,183-188 count as
    "nnz_all"; sorted row-major, ready for AbhsfMatrix.from_elements.  A
    general matrix comes back unchanged."""
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    vals = np.asarray(vals, np.float64)
    if symmetry == "general":
        return rows, cols, vals
    if symmetry not in ("symmetric", "skew", "hermitian"):
        raise ValueError("symmetry: general, symmetric, skew or hermitian")
    off = rows != cols
    mv = -vals[off] if symmetry == "skew" else vals[off]
    r = np.concatenate([rows, cols[off]])
    c = np.concatenate([cols, rows[off]])
    v = np.concatenate([vals, mv])
    order = np.lexsort((c, r))
    return r[order], c[order], v[order]


def read_mm(path: str):
    """A binary .mm matrix file (the layout utils/mtx2mm/mtx2mm.cpp:102-135
    writes), returned as read_mtx returns the text file it was made from."""
    c = capi.CooHost()
    capi.check(capi.lib.abhsf_read_mm(os.fsencode(path), C.byref(c)))
    return _coo_result(c)


def write_mm(path: str, rows, cols, vals, m: int, n: int, matrix_type: str = "real",
             symmetry: str = "general") -> None:
    """Writes 0-based COO arrays as a binary .mm file (vals ignored for a
    "binary" matrix)."""
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    cols = np.ascontiguousarray(cols, dtype=np.int64)
    if rows.shape != cols.shape or rows.ndim != 1:
        raise capi.InvalidValue(capi.INVALID_VALUE, "rows and cols must be 1-D arrays of one length")
    if matrix_type not in ("real", "binary") or symmetry not in _SYMMETRIES:
        raise capi.InvalidValue(capi.INVALID_VALUE, "matrix_type real / binary; symmetry " + " / ".join(_SYMMETRIES))
    c = capi.CooHost()
    c.m, c.n, c.nnz = int(m), int(n), rows.size
    c.matrix_type = capi.MATRIX_TYPES[matrix_type]
    c.symmetry = _SYMMETRIES.index(symmetry)
    c.rows = rows.ctypes.data_as(C.POINTER(C.c_int64))
    c.cols = cols.ctypes.data_as(C.POINTER(C.c_int64))
    if matrix_type == "real":
        vals = np.ascontiguousarray(vals, dtype=np.float64)
        if vals.shape != rows.shape:
            raise capi.InvalidValue(capi.INVALID_VALUE, "vals must have one value per element")
        c.vals = vals.ctypes.data_as(C.POINTER(C.c_double))
    capi.check(capi.lib.abhsf_write_mm(os.fsencode(path), C.byref(c)))


def mtx2mm(src: str, dst: str, threads: int = 0) -> None:
    """Converts a Matrix Market file to the binary .mm layout (what
    utils/mtx2mm does, after read_mtx's zero-drop)."""
    rows, cols, vals, m, n, info = read_mtx(src, threads)
    write_mm(dst, rows, cols, vals, m, n, info["matrix_type"], info["symmetry"])


def mmf_line(m: int, n: int, nnz: int, matrix_type: str | int, r: int, s: int, hist: dict[int, int]):
    """One line of the reference's mmf-single / mmf-double
    (block_statistics/mmf.cpp:53-138): [coo32, csr32, coo, csr, bitmap, dense,
    abhsf, abhsf134], values included."""
    mt = capi.MATRIX_TYPES[matrix_type] if isinstance(matrix_type, str) else int(matrix_type)
    h = np.zeros((max(hist) + 1) if hist else 1, dtype=np.uint64)
    for z, c in hist.items():
        h[z] = c
    o1 = np.zeros(8, dtype=np.uint64)
    o2 = np.zeros(8, dtype=np.uint64)
    capi.check(capi.lib.abhsf_mmf_line(m, n, nnz, mt, r, s, h.ctypes.data_as(capi._u64p), h.size,
                                       o1.ctypes.data_as(capi._u64p), o2.ctypes.data_as(capi._u64p)))
    return [int(v) for v in o1], [int(v) for v in o2]


def block_scheme_bits(scheme, r: int, s: int, nnz: int, bits_per_value: int = 64) -> int:
    sc = capi.SCHEME_NAMES.index(scheme) if isinstance(scheme, str) else int(scheme)
    return int(capi.lib.abhsf_block_scheme_bits(sc, r, s, nnz, bits_per_value))


def block_select_scheme(r: int, s: int, nnz: int, bits_per_value: int = 64, is_binary: bool = False,
                        allow_csr: bool = True) -> str:
    return capi.SCHEME_NAMES[capi.lib.abhsf_block_select_scheme(r, s, nnz, bits_per_value, int(is_binary),
                                                                int(allow_csr))]


def _info(i: "capi.CgInfo") -> dict:
    return {"iterations": int(i.iterations), "outer_iterations": int(i.outer_iterations),
            "converged": bool(i.converged), "rel_residual": float(i.rel_residual)}


def _solver_vectors(A, b, x):
    if not (_is_cuda(b) and _is_cuda(x)):
        raise capi.InvalidValue(capi.INVALID_VALUE, "b and x must be CUDA tensors")
    if b.dtype != torch.float64 or x.dtype != torch.float64 or b.numel() != A.n or x.numel() != A.n:
        raise capi.InvalidValue(capi.INVALID_VALUE, f"b and x must be float64 with n={A.n} entries")
    if not (b.is_contiguous() and x.is_contiguous()):
        raise capi.InvalidValue(capi.INVALID_VALUE, "b and x must be contiguous")


def cg(A: AbhsfMatrix, b, x, rtol: float = 1e-10, max_iters: int = 100000, stream=None) -> dict:
    """Solves A x = b (A SPD, f64) by FP64 conjugate gradients; x (CUDA
    float64) is the initial guess and receives the solution."""
    A._check_open()
    _solver_vectors(A, b, x)
    info = capi.CgInfo()
    capi.check(capi.lib.abhsf_cg(A._h, b.data_ptr(), x.data_ptr(), float(rtol), int(max_iters), C.byref(info),
                                 _stream_ptr(stream)))
    return _info(info)


def cg_mixed(A64: AbhsfMatrix, A_lo: AbhsfMatrix, b, x, rtol: float = 1e-10, max_iters: int = 100000,
             update_factor: float = 1e-1, max_updates: int = 1000, stream=None) -> dict:
    """Solves A x = b by an f32 CG on A_lo (the same matrix stored as f32 or
    bf16) whose solution accumulates in FP64 and whose residual is replaced
    by the FP64 residual of A64 each time it falls by update_factor."""
    A64._check_open()
    A_lo._check_open()
    _solver_vectors(A64, b, x)
    info = capi.CgInfo()
    capi.check(capi.lib.abhsf_cg_mixed(A64._h, A_lo._h, b.data_ptr(), x.data_ptr(), float(rtol), int(max_iters),
                                       float(update_factor), int(max_updates), C.byref(info), _stream_ptr(stream)))
    return _info(info)


class AbhsfBatch:
    """Several f64 matrices of one block size whose SpMVs run as one
    kernel launch (abhsf_batch_*).  Keeps the matrices alive."""

    def __init__(self, mats, stream=None):
        self._mats = list(mats)
        for a in self._mats:
            a._check_open()
        arr = (C.c_void_p * len(self._mats))(*[a._h.value for a in self._mats])
        self._h = C.c_void_p()
        capi.check(capi.lib.abhsf_batch_create(arr, len(self._mats), _stream_ptr(stream), C.byref(self._h)))

    def pointer_tables(self, xs, ys):
        """Device int64 tensors with the data pointers of xs and ys (CUDA
        float64 vectors of n_i and m_i entries), for spmv_tables."""
        if len(xs) != len(self._mats) or len(ys) != len(self._mats):
            raise capi.InvalidValue(capi.INVALID_VALUE, "one x and one y per matrix")
        for a, x, y in zip(self._mats, xs, ys):
            if not (_is_cuda(x) and _is_cuda(y)) or x.dtype != torch.float64 or y.dtype != torch.float64:
                raise capi.InvalidValue(capi.INVALID_VALUE, "x and y must be CUDA float64 tensors")
            if x.numel() != a.n or y.numel() != a.m or not (x.is_contiguous() and y.is_contiguous()):
                raise capi.InvalidValue(capi.INVALID_VALUE, "x_i / y_i must be contiguous with n_i / m_i entries")
        px = torch.tensor([x.data_ptr() for x in xs], dtype=torch.int64, device=xs[0].device)
        py = torch.tensor([y.data_ptr() for y in ys], dtype=torch.int64, device=ys[0].device)
        return px, py

    def spmv_tables(self, px, py, stream=None) -> None:
        """y_i += A_i x_i with device pointer tables (graph-capturable)."""
        capi.check(capi.lib.abhsf_batch_spmv(self._h, px.data_ptr(), py.data_ptr(), _stream_ptr(stream)))

    def spmv(self, xs, ys, stream=None) -> None:
        """y_i += A_i x_i for every matrix, one launch."""
        px, py = self.pointer_tables(xs, ys)
        self.spmv_tables(px, py, stream)
        self._keep = (px, py)  # until the next call: the launch reads them asynchronously

    def status(self, clear: bool = False, stream=None) -> int:
        v = C.c_int32()
        capi.check(capi.lib.abhsf_batch_status(self._h, _stream_ptr(stream), int(clear), C.byref(v)))
        return int(v.value)

    def launches(self) -> int:
        """Kernels one spmv launches (the tile kernel, the row-slice kernel,
        the chain kernel: those the batch's matrices need)."""
        v = C.c_int32()
        capi.check(capi.lib.abhsf_batch_kernels(self._h, C.byref(v)))
        return int(v.value)

    def release(self) -> None:
        if self._h is not None and self._h.value:
            capi.check(capi.lib.abhsf_batch_release(self._h))
        self._h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass
