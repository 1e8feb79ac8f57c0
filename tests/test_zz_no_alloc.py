"""abhsf_block_histogram_noalloc: the GPU block histogram for callers that may
not allocate device memory (their memory belongs to their own allocator or
pool, a cudaMalloc could synchronise the device at a bad moment, or they run
at their memory limit).  All its scratch is a fixed array inside the library.

Checked through the C ABI against the allocating abhsf_block_histogram, on
consecutive calls that reuse the scratch, including one near the size limit.
Collected last (file name) so that a failure here cannot hide another test.
"""
import ctypes as C

import numpy as np
import pytest

from abhsf_b200 import capi
from abhsf_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _histograms(coo, r, s):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    rows = torch.from_numpy(coo.rows).cuda()
    cols = torch.from_numpy(coo.cols).cuda()
    out = []
    for fn in ("abhsf_block_histogram", "abhsf_block_histogram_noalloc"):
        hist = np.zeros(r * s + 1, dtype=np.uint64)
        blocks = C.c_int64(-1)
        if fn == "abhsf_block_histogram":
            st = capi.lib.abhsf_block_histogram(rows.data_ptr(), cols.data_ptr(), coo.nnz, coo.m, coo.n, r, s, 1,
                                                stream, hist.ctypes.data_as(capi._u64p), hist.size, C.byref(blocks))
        else:
            st = capi.lib.abhsf_block_histogram_noalloc(rows.data_ptr(), cols.data_ptr(), coo.nnz, coo.m, coo.n, r,
                                                        s, stream, hist.ctypes.data_as(capi._u64p), hist.size,
                                                        C.byref(blocks))
        capi.check(st)
        out.append((hist, blocks.value))
    return out


def test_noalloc_histogram_equals_allocating_histogram_on_consecutive_calls(gpu):
    cases = [
        (W.random_blocky(4000, 5000, 64, 300, seed=41), 64, 64),
        (W.random_uniform(3000, 3500, capi.NOALLOC_MAX_NNZ - 1000, seed=42), 8, 32),  # near the limit
        (W.laplacian_2d(256), 256, 2),
    ]
    for coo, r, s in cases:
        assert 0 < coo.nnz <= capi.NOALLOC_MAX_NNZ
        (h_ref, b_ref), (h_new, b_new) = _histograms(coo, r, s)
        np.testing.assert_array_equal(h_new, h_ref)
        assert b_new == b_ref > 0
        assert int((h_ref * np.arange(h_ref.size, dtype=np.uint64)).sum()) == coo.nnz


def test_noalloc_histogram_makes_no_device_allocation(gpu):
    """After its first call on the device (which looks up the scratch array's
    address), a call makes no cudaMalloc inside the library and leaves the
    device's free memory as it was: the property the entry point exists for."""
    import torch
    coo = W.random_blocky(4000, 5000, 64, 300, seed=43)
    stream = torch.cuda.current_stream().cuda_stream
    rows = torch.from_numpy(coo.rows).cuda()
    cols = torch.from_numpy(coo.cols).cuda()
    hist = np.zeros(64 * 64 + 1, dtype=np.uint64)

    def call():
        capi.check(capi.lib.abhsf_block_histogram_noalloc(rows.data_ptr(), cols.data_ptr(), coo.nnz, coo.m, coo.n,
                                                          64, 64, stream, hist.ctypes.data_as(capi._u64p),
                                                          hist.size, None))

    call()  # set-up on this device
    torch.cuda.synchronize()
    before = capi.lib.abhsf_test_device_allocations()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    assert capi.lib.abhsf_test_device_allocations() == before
    assert torch.cuda.mem_get_info()[0] == free_before
    # the counter does see the allocating histogram's scratch
    blocks = C.c_int64(-1)
    capi.check(capi.lib.abhsf_block_histogram(rows.data_ptr(), cols.data_ptr(), coo.nnz, coo.m, coo.n, 64, 64, 1,
                                              stream, hist.ctypes.data_as(capi._u64p), hist.size, C.byref(blocks)))
    assert capi.lib.abhsf_test_device_allocations() > before


def test_noalloc_histogram_rejects_inputs_beyond_its_limit(gpu):
    import torch
    n = capi.NOALLOC_MAX_NNZ + 1
    rows = torch.zeros(n, dtype=torch.int64, device="cuda")
    hist = np.zeros(5, dtype=np.uint64)
    st = capi.lib.abhsf_block_histogram_noalloc(rows.data_ptr(), rows.data_ptr(), n, 10, 10, 2, 2, None,
                                                hist.ctypes.data_as(capi._u64p), hist.size, None)
    assert st == capi.INVALID_VALUE
    assert b"ABHSF_NOALLOC_MAX_NNZ" in capi.lib.abhsf_last_error_string()
