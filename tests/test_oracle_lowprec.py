"""The oracle's f32 / bf16 value conversion and f32 SpMV loop (the checkers
of the GPU f32 SpMV), against numpy's own rounding."""
import numpy as np

from oracle import oracle


def _bf16_numpy(v):
    """RNE of the f32 value to its upper 16 bits (finite inputs)."""
    u = np.asarray(v, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint32) << 16
    return r.astype(np.uint32).view(np.float32)


def test_values_as_f32_matches_numpy_rounding():
    v = np.random.default_rng(0).standard_normal(20000) * np.exp(np.random.default_rng(1).uniform(-20, 20, 20000))
    np.testing.assert_array_equal(oracle.values_as_f32(v, "f32"), v.astype(np.float32))
    np.testing.assert_array_equal(oracle.values_as_f32(v, "bf16"), _bf16_numpy(v))
    # ties to even at the bf16 boundary: 1 + 2^-8 is halfway between 1 and 1 + 2^-7
    np.testing.assert_array_equal(oracle.values_as_f32(np.array([1 + 2.0**-8, 1 + 3 * 2.0**-8]), "bf16"),
                                  np.array([1.0, 1 + 2.0**-6], dtype=np.float32))


def test_spmv_elements_f32_matches_sequential_numpy():
    rng = np.random.default_rng(3)
    rows = np.sort(rng.integers(0, 50, 400))
    cols = rng.integers(0, 60, 400)
    vals = rng.standard_normal(400).astype(np.float32)
    x = rng.uniform(-1, 1, 60).astype(np.float32)
    y0 = rng.standard_normal(50).astype(np.float32)
    want = y0.copy()
    for r, c, v in zip(rows, cols, vals):
        want[r] = np.float32(want[r] + np.float32(v * x[c]))
    np.testing.assert_array_equal(oracle.spmv_elements_f32(rows, cols, vals, x, y0), want)
