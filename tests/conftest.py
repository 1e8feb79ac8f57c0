import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# y += A x must match the FP64 oracle within this bound per element, relative to
# the magnitude of the terms summed into it: |dy_i| <= RTOL * ((|A||x|)_i + |y0_i|).
# Plain |dy_i| / |y_i| is also reported; it is undefined where y_i cancels to ~0.
SPMV_RTOL = 1e-13


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def golden_stats() -> dict:
    with open(os.path.join(GOLDEN, "block_stats.json")) as f:
        return json.load(f)


def golden_matrices():
    """name -> Coo for the small golden matrices."""
    from abhsf_b200.workloads import Coo
    z = np.load(os.path.join(GOLDEN, "matrices.npz"))
    names = sorted({k.split("__")[0] for k in z.files})
    out = {}
    for nm in names:
        m, n = (int(v) for v in z[nm + "__shape"])
        out[nm] = Coo(z[nm + "__rows"], z[nm + "__cols"], z[nm + "__vals"], m, n, nm)
    return out


def golden_spmv() -> dict:
    z = np.load(os.path.join(GOLDEN, "spmv_ref.npz"))
    return {k: z[k] for k in z.files}


def assert_spmv_close(y, y_ref, scale, rtol=SPMV_RTOL):
    """|y - y_ref| <= rtol * scale elementwise; returns the worst ratios."""
    y = np.asarray(y)
    err = np.abs(y - y_ref)
    bound = rtol * scale
    bad = np.nonzero(err > bound)[0]
    assert bad.size == 0, (f"{bad.size} elements out of tolerance, first {bad[:5]}: "
                           f"y={y[bad[:5]]} ref={y_ref[bad[:5]]} scale={scale[bad[:5]]}")
    nz = scale > 0
    worst_scaled = float(np.max(err[nz] / scale[nz])) if nz.any() else 0.0
    big = np.abs(y_ref) > 1e-8 * np.maximum(scale, 1e-300)
    worst_rel = float(np.max(err[big] / np.abs(y_ref[big]))) if big.any() else 0.0
    return worst_scaled, worst_rel


@pytest.fixture(scope="session")
def gpu():
    import torch
    assert torch.cuda.is_available()
    torch.cuda.init()
    return torch.device("cuda:0")
