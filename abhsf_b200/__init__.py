"""abhsf_b200: B200-native (sm_100a) builder and SpMV for the Adaptive-Blocking
Hierarchical Storage Format.  The compute path is libabhsf_b200.so (CUDA C++,
C ABI in include/abhsf/abhsf_gpu.h); this package is its Python binding.

The binding is loaded on first use of a public name, so that
``python -m abhsf_b200.build`` works before the library exists."""
import importlib

_EXPORTS = {
    "AbhsfError": "capi", "DuplicateEntry": "capi", "IndexOutOfRange": "capi", "InvalidValue": "capi",
    "Unsupported": "capi",
    "AbhsfMatrix": "matrix", "AbhsfBatch": "matrix", "block_histogram": "matrix", "read_mtx": "matrix",
    "read_mtx_device": "matrix",
    "read_mm": "matrix", "write_mm": "matrix", "mtx2mm": "matrix", "expand_symmetric": "matrix", "block_histograms_all": "matrix", "block_scheme_bits": "matrix",
    "block_select_scheme": "matrix", "mmf_line": "matrix", "cg": "matrix", "cg_mixed": "matrix",
    "ShardedMatrix": "sharded",
}

__all__ = sorted(_EXPORTS)


def __getattr__(name):
    mod = _EXPORTS.get(name)
    if mod is None:
        raise AttributeError(f"module 'abhsf_b200' has no attribute {name!r}")
    return getattr(importlib.import_module(f".{mod}", __name__), name)
