"""ctypes binding of the C ABI in include/abhsf/abhsf_gpu.h.

Loads the in-tree abhsf_b200/libabhsf_b200.so.  There is no fallback: if the
library is missing, importing this module raises, naming the build command.
"""
from __future__ import annotations

import ctypes as C
import os
import re

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libabhsf_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "abhsf", "abhsf_gpu.h")

SUCCESS, INVALID_VALUE, INDEX_OUT_OF_RANGE, DUPLICATE_ENTRY, OUT_OF_MEMORY, UNSUPPORTED, CUDA_ERROR = range(7)
SCHEME_COO, SCHEME_CSR, SCHEME_BITMAP, SCHEME_DENSE = range(4)
SCHEME_NAMES = ("coo", "csr", "bitmap", "dense")
VALUE_TYPES = {"f64": 0, "f32": 1, "bf16": 2}
MATRIX_TYPES = {"binary": 0, "integer": 1, "real": 2, "complex": 3}
SUM_ORDERS = {"reference": 0, "tree": 1}
NOALLOC_MAX_NNZ = 1048576
BSTATS_ALL_LEN = 260164
DEVSTAT_WAIT_TIMEOUT = 1
SELECTORS = {"minbss": 0, "learned": 1, "autotune": 2, "learned_time": 3}
FEATURES, MLP_HIDDEN, MLP_CLASSES = 12, 64, 5
MLP_PARAMS = (FEATURES * MLP_HIDDEN + MLP_HIDDEN + MLP_HIDDEN * MLP_HIDDEN + MLP_HIDDEN +
              MLP_HIDDEN * MLP_CLASSES + MLP_CLASSES + 2 * FEATURES)
BLOCK_SIZES = (16, 32, 64, 128, 256)


class AbhsfError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"abhsf status {status}: {msg}")
        self.status = status


class InvalidValue(AbhsfError, ValueError):
    pass


class IndexOutOfRange(AbhsfError, IndexError):
    pass


class DuplicateEntry(AbhsfError, ValueError):
    pass


class OutOfMemory(AbhsfError, MemoryError):
    pass


class Unsupported(AbhsfError, NotImplementedError):
    pass


class CudaError(AbhsfError):
    pass


_ERR = {INVALID_VALUE: InvalidValue, INDEX_OUT_OF_RANGE: IndexOutOfRange, DUPLICATE_ENTRY: DuplicateEntry,
        OUT_OF_MEMORY: OutOfMemory, UNSUPPORTED: Unsupported, CUDA_ERROR: CudaError}


class BuildOpts(C.Structure):
    _fields_ = [("block_size", C.c_int32), ("value_type", C.c_int32), ("allow_csr", C.c_int32),
                ("matrix_type", C.c_int32), ("forced_scheme", C.c_int32), ("inputs_on_device", C.c_int32),
                ("sum_order", C.c_int32), ("bits_per_value", C.c_int64), ("selector", C.c_int32),
                ("slice_tile_nnz", C.c_int32), ("selector_model", C.c_void_p)]


class CooHost(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("nnz", C.c_int64), ("matrix_type", C.c_int32),
                ("symmetry", C.c_int32), ("stored_triangle", C.c_int32), ("reserved", C.c_int32),
                ("rows", C.POINTER(C.c_int64)), ("cols", C.POINTER(C.c_int64)), ("vals", C.POINTER(C.c_double))]


class CooDevice(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("nnz", C.c_int64), ("matrix_type", C.c_int32),
                ("symmetry", C.c_int32), ("stored_triangle", C.c_int32), ("reserved", C.c_int32),
                ("rows", C.c_void_p), ("cols", C.c_void_p), ("vals", C.c_void_p), ("host_parsed", C.c_int64)]


class CgInfo(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("outer_iterations", C.c_int32), ("converged", C.c_int32),
                ("reserved", C.c_int32), ("rel_residual", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("m", C.c_int64), ("n", C.c_int64), ("nnz", C.c_int64),
                ("block_size", C.c_int32), ("value_type", C.c_int32),
                ("block_rows", C.c_int64), ("block_cols", C.c_int64), ("tiles", C.c_int64),
                ("tiles_per_scheme", C.c_int64 * 4), ("nnz_per_scheme", C.c_int64 * 4),
                ("stored_values", C.c_int64), ("payload_bytes", C.c_int64), ("format_bytes", C.c_int64),
                ("msmf_bits", C.c_uint64 * 8), ("spmv_bytes", C.c_int64)]


_vp = C.c_void_p
_i64 = C.c_int64
_i32 = C.c_int32
_u64p = C.POINTER(C.c_uint64)
_fp = C.POINTER(C.c_float)

# name -> (restype, argtypes)
PROTOTYPES = {
    "abhsf_abi_version": (_i32, []),
    "abhsf_device_status": (C.c_int, [_vp, _vp, _i32, C.POINTER(_i32)]),
    "abhsf_test_set_hooks": (None, [_i64, C.c_uint32]),
    "abhsf_test_ring_variant": (C.c_int, [_vp, _i32, C.POINTER(_i32), C.POINTER(_i32)]),
    "abhsf_test_device_allocations": (_i64, []),
    "abhsf_slices_info": (C.c_int, [_vp] + [C.POINTER(_i64)] * 5),
    "abhsf_batch_kernels": (C.c_int, [_vp, C.POINTER(_i32)]),
    "abhsf_spmv_kernels": (C.c_int, [_vp, C.POINTER(_i32)]),
    "abhsf_slices_export": (C.c_int, [_vp] * 10),
    "abhsf_last_error_string": (C.c_char_p, []),
    "abhsf_build_opts_default": (None, [C.POINTER(BuildOpts)]),
    "abhsf_build": (C.c_int, [_vp, _vp, _vp, _i64, _i64, _i64, C.POINTER(BuildOpts), _vp, C.POINTER(_vp)]),
    "abhsf_spmv": (C.c_int, [_vp, _vp, _vp, _vp]),
    "abhsf_spmv_host": (C.c_int, [_vp, _vp, _vp, _vp]),
    "abhsf_spmm": (C.c_int, [_vp, _i32, _vp, _i64, _vp, _i64, _vp]),
    "abhsf_spmv_f32": (C.c_int, [_vp, _vp, _vp, _vp]),
    "abhsf_batch_create": (C.c_int, [_vp, _i32, _vp, C.POINTER(_vp)]),
    "abhsf_batch_spmv": (C.c_int, [_vp, _vp, _vp, _vp]),
    "abhsf_batch_status": (C.c_int, [_vp, _vp, _i32, C.POINTER(_i32)]),
    "abhsf_batch_release": (C.c_int, [_vp]),
    "abhsf_cg": (C.c_int, [_vp, _vp, _vp, C.c_double, _i32, C.POINTER(CgInfo), _vp]),
    "abhsf_cg_mixed": (C.c_int, [_vp, _vp, _vp, _vp, C.c_double, _i32, C.c_double, _i32, C.POINTER(CgInfo),
                                 _vp]),
    "abhsf_release": (C.c_int, [_vp]),
    "abhsf_stats_get": (C.c_int, [_vp, C.POINTER(Stats)]),
    "abhsf_export_host": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "abhsf_block_histogram": (C.c_int, [_vp, _vp, _i64, _i64, _i64, _i32, _i32, _i32, _vp, _u64p, _i64,
                                        C.POINTER(_i64)]),
    "abhsf_block_histogram_all": (C.c_int, [_vp, _vp, _i64, _i64, _i64, _i32, _vp, _u64p, C.POINTER(_i64)]),
    "abhsf_block_histogram_noalloc": (C.c_int, [_vp, _vp, _i64, _i64, _i64, _i32, _i32, _vp, _u64p, _i64,
                                                C.POINTER(_i64)]),
    "abhsf_mmf_line": (C.c_int, [_i64, _i64, _i64, _i32, _i32, _i32, _u64p, _i64, _u64p, _u64p]),
    "abhsf_block_size_storage": (C.c_int, [_vp, _vp, _i64, _i64, _i64, C.POINTER(BuildOpts), _vp, _u64p,
                                           C.POINTER(_i32)]),
    "abhsf_autotune": (C.c_int, [_vp, _vp, _vp, _i64, _i64, _i64, C.POINTER(BuildOpts), _i32, _i32, _vp, _fp,
                                 C.POINTER(_i32), C.POINTER(_vp)]),
    "abhsf_selector_features": (C.c_int, [_vp, _vp, _i64, _i64, _i64, _i32, _vp, _fp]),
    "abhsf_selector_predict": (C.c_int, [_vp, _fp, _vp, C.POINTER(_i32)]),
    "abhsf_selector_builtin_model": (C.c_int, [_fp]),
    "abhsf_selector_builtin_time_model": (C.c_int, [_fp]),
    "abhsf_mlp_forward": (C.c_int, [_vp, _vp, _i32, _vp, _vp, _vp]),
    "abhsf_mlp_backward": (C.c_int, [_vp, _vp, _vp, _i32, _vp, _vp, _vp, _vp, _vp, _vp]),
    "abhsf_mlp_adam": (C.c_int, [_vp, _vp, _vp, _vp, _i32, C.c_float, _vp]),
    "abhsf_read_mtx": (C.c_int, [C.c_char_p, _i32, C.POINTER(CooHost)]),
    "abhsf_read_mtx_device": (C.c_int, [C.c_char_p, C.c_void_p, C.POINTER(CooDevice)]),
    "abhsf_coo_device_free": (C.c_int, [C.POINTER(CooDevice)]),
    "abhsf_coo_device_copy": (C.c_int, [C.POINTER(CooDevice), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "abhsf_test_parse_decimal": (_i32, [C.c_char_p, _i64, C.POINTER(C.c_double), C.POINTER(_i64)]),
    "abhsf_read_mm": (C.c_int, [C.c_char_p, C.POINTER(CooHost)]),
    "abhsf_write_mm": (C.c_int, [C.c_char_p, C.POINTER(CooHost)]),
    "abhsf_coo_host_free": (C.c_int, [C.POINTER(CooHost)]),
    "abhsf_block_scheme_bits": (C.c_uint64, [_i32, _i64, _i64, _i64, _i64]),
    "abhsf_block_select_scheme": (_i32, [_i64, _i64, _i64, _i64, _i32, _i32]),
}


def header_functions(path: str = HEADER) -> list[str]:
    """Names of the functions include/abhsf/*.h declares with ABHSF_API."""
    names = []
    hdir = os.path.dirname(path)
    for fn in sorted(os.listdir(hdir)):
        if fn.endswith(".h"):
            names += re.findall(r"ABHSF_API[^;(]*?\b(abhsf_\w+)\s*\(", open(os.path.join(hdir, fn)).read())
    return names


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m abhsf_b200.build` "
                          "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    return L


lib = _load()


def check(status: int) -> None:
    if status != SUCCESS:
        msg = lib.abhsf_last_error_string().decode(errors="replace")
        raise _ERR.get(status, AbhsfError)(status, msg)
