"""abhsf_b200: B200-native (sm_100a) builder and SpMV for the Adaptive-Blocking
Hierarchical Storage Format.  The compute path is libabhsf_b200.so (CUDA C++,
C ABI in include/abhsf/abhsf_gpu.h); this package is its Python binding."""
from .capi import AbhsfError, DuplicateEntry, IndexOutOfRange, InvalidValue, Unsupported  # noqa: F401
from .matrix import (AbhsfMatrix, block_histogram, block_scheme_bits, block_select_scheme,  # noqa: F401
                     mmf_line)
