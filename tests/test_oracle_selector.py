"""The block-size selector on the CPU: the oracle's min-bss sweep against the
reference's own mmf output, the oracle's MLP gradients against finite
differences, and the host logic (regret, targets, the model file)."""
import numpy as np
import pytest

from conftest import golden_matrices, golden_stats
from abhsf_b200 import capi
from abhsf_b200 import selector as sel
from abhsf_b200 import workloads as W
from oracle import oracle
from oracle import selector_oracle as so

STATS = golden_stats()
MATS = golden_matrices()


def _coo(name):
    return W.laplacian_2d(512) if name == "laplace2d_512" else MATS[name]


@pytest.mark.parametrize("name", sorted(STATS))
def test_oracle_min_bss_matches_reference_mmf(name):
    """min-bss over the square sizes: the abhsf / abhsf134 columns of the
    reference's mmf-double lines (block_statistics/min-bss.cpp:14-58)."""
    g = STATS[name]
    m, n, _, _, _, mtype, _ = g["props"]
    coo = _coo(name)
    lines = {(l[0], l[1]): l[2:] for l in g["mmf_double"]}
    for allow_csr, col in ((True, 6), (False, 7)):
        bits, best = so.block_size_storage(coo.rows, coo.cols, m, n, mtype, allow_csr)
        want = [lines[(s, s)][col] for s in so.SIZES]
        assert bits.tolist() == want
        assert best == so.SIZES[int(np.argmin(want))]


def test_oracle_features_known_answer():
    # 2 x 3 grid of 64-tiles; rows 0..99 diagonal plus one far element
    rows = np.r_[np.arange(100), 5]
    cols = np.r_[np.arange(100), 150]
    f = so.features(rows, cols, 128, 192)
    assert f[0] == 7 and np.isclose(f[1], np.log2(192))
    assert np.isclose(f[2], np.log2(101 / 128 + 1))
    cnt = np.bincount(rows, minlength=128)
    assert np.isclose(f[3], np.log2(cnt.std() + 1))
    assert np.isclose(f[4], 145 / 192) and np.isclose(f[5], 145 / 101 / 192)
    # tiles: (0,0) 64 nnz, (1,1) 36 nnz, (0,2) 1 nnz
    assert np.allclose(f[6:11], [1 / 101, 0, 100 / 101, 0, 0])
    assert np.isclose(f[11], np.log2(3 / 2 + 1))


def _rand_params(seed):
    rng = np.random.default_rng(seed)
    p = rng.standard_normal(so.P) * 0.3
    p[so.OMEAN:so.OISTD] = rng.standard_normal(so.F) * 0.1
    p[so.OISTD:] = rng.uniform(0.5, 2.0, so.F)
    return p


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = _rand_params(2)
    X = rng.standard_normal((7, so.F))
    T = sel.targets_from_bits(rng.integers(100, 200, (7, 5)).astype(np.uint64), tau=0.1).astype(np.float64)
    g, _ = so.backward(p, X, T)
    idx = np.r_[rng.choice(so.OMEAN, 60, replace=False), so.OB3, so.OB3 + 4, so.OW3, so.OB1]
    for q in idx:
        e = np.zeros(so.P)
        e[q] = 1e-6
        fd = (so.loss(p + e, X, T) - so.loss(p - e, X, T)) / 2e-6
        assert abs(fd - g[q]) <= 1e-6 + 1e-5 * abs(fd), q
    assert np.all(g[so.OMEAN:] == 0)


def test_regret_metric():
    bits = np.array([[100, 110, 150, 200, 300], [90, 80, 80, 95, 99]], np.uint64)
    r = sel.regret(bits, np.array([1, 0]))
    assert np.allclose(r, [10.0, 12.5])
    s = sel.regret_summary(bits, np.array([0, 2]))
    assert s == {"avg_pct": 0.0, "max_pct": 0.0, "exact": 1.0}
    s = sel.regret_summary(bits, np.array([1, 0]))
    assert np.isclose(s["avg_pct"], 11.25) and np.isclose(s["max_pct"], 12.5) and s["exact"] == 0.0


def test_targets_from_bits():
    bits = np.array([[100, 110, 100, 200, 300]], np.uint64)
    t0 = sel.targets_from_bits(bits)
    assert t0.tolist() == [[1, 0, 0, 0, 0]]  # ties to the smaller size
    t = sel.targets_from_bits(bits, tau=0.05)
    assert np.isclose(t.sum(), 1) and np.isclose(t[0, 0], t[0, 2]) and t[0, 1] < t[0, 0] and t[0, 4] < 1e-6


def test_model_include_round_trip(tmp_path):
    p = _rand_params(3).astype(np.float32)
    path = tmp_path / "m.inc"
    sel.write_model_inc(p, str(path))
    body = path.read_text().split("{", 1)[1].split("}", 1)[0]
    back = np.array([float(v.strip().rstrip("f")) for v in body.split(",") if v.strip()], np.float32)
    assert back.size == capi.MLP_PARAMS and np.array_equal(back, p)


def test_builtin_model_is_exported():
    p = sel.builtin_model()
    assert p.shape == (capi.MLP_PARAMS,) and np.all(np.isfinite(p))
    assert np.all(p[so.OISTD:] > 0)


def test_parameter_count_matches_header():
    assert capi.MLP_PARAMS == so.P == 5341


def test_builtin_model_regret_on_heldout_fixture():
    """The shipped model on the 200 held-out matrices of its training run
    (tests/golden/selector_heldout.npz, written by
    `python -m abhsf_b200.selector train`): forward pass in the float64
    oracle, regret as block_statistics/consistency.cpp:147-173 computes it,
    against every fixed block size."""
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "selector_heldout.npz"))
    X, bits = z["X"], z["bits"]
    assert X.shape == (200, 12) and bits.shape == (200, 5)
    probs, _ = so.forward(sel.builtin_model(), X)
    learned = sel.regret_summary(bits, probs.argmax(axis=1))
    fixed = [sel.regret_summary(bits, np.full(len(X), k)) for k in range(5)]
    assert learned["avg_pct"] < 0.1 * min(f["avg_pct"] for f in fixed), (learned, fixed)
    assert learned["max_pct"] < min(f["max_pct"] for f in fixed)
    assert learned["exact"] >= 0.9


def test_builtin_time_model_on_heldout_fixture():
    """The model trained on measured SpMV time, on the 300 held-out matrices
    of its training run (tests/golden/selector_time_heldout.npz, written by
    `python -m abhsf_b200.selector train-time`: features, storage and the
    FP64 SpMV time at each size, timed on a B200): forward pass in the
    float64 oracle.  Its choices are faster in total than min-bss's and than
    every fixed size's, and its time regret (the consistency.cpp:147-173
    measure with time in place of storage) is below theirs on average."""
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "selector_time_heldout.npz"))
    X, bits, ms = z["X"], z["bits"], z["ms"]
    assert X.shape == (300, 12) and bits.shape == (300, 5) and ms.shape == (300, 5)
    assert np.all(ms > 0)
    probs, _ = so.forward(sel.builtin_time_model(), X)
    learned = sel.time_regret_summary(ms, probs.argmax(axis=1))
    minbss = sel.time_regret_summary(ms, bits.astype(np.float64).argmin(axis=1))
    fixed = [sel.time_regret_summary(ms, np.full(len(X), k)) for k in range(5)]
    assert learned["total_over_best"] < minbss["total_over_best"], (learned, minbss)
    assert learned["total_over_best"] < min(f["total_over_best"] for f in fixed), (learned, fixed)
    assert learned["avg_pct"] < min([minbss["avg_pct"]] + [f["avg_pct"] for f in fixed])
    # the storage model picks by storage; its choices are no faster than min-bss's
    store = sel.time_regret_summary(ms, so.forward(sel.builtin_model(), X)[0].argmax(axis=1))
    assert store["total_over_best"] > learned["total_over_best"]
