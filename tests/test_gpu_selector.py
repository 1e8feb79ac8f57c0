"""GPU block-size selection: the exhaustive sweep (abhsf_block_size_storage)
bit-exact against the oracle, the selector's features, the MLP's forward,
backward and Adam kernels against the float64 oracle, abhsf_build with
block_size 0, and what the shipped model gains over a fixed block size."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden_matrices, golden_stats
from abhsf_b200 import AbhsfMatrix, capi
from abhsf_b200 import selector as sel
from abhsf_b200 import workloads as W
from oracle import selector_oracle as so

pytestmark = pytest.mark.gpu

# float32 kernels against the float64 oracle
FEAT_TOL = dict(rtol=2e-6, atol=2e-6)
PROB_TOL = dict(rtol=1e-5, atol=1e-6)
GRAD_TOL = dict(rtol=1e-4, atol=1e-6)


def _small(seed, n_max=60_000):
    r, c, m, n, name = W.selector_matrix(seed, n_min=2_000, n_max=n_max, nnz_max=1_500_000, device="cpu")
    return r.numpy(), c.numpy(), m, n, name


@pytest.mark.parametrize("name", sorted(golden_stats()))
def test_sweep_matches_oracle_on_golden(gpu, name):
    g = golden_stats()[name]
    m, n, _, _, _, mtype, _ = g["props"]
    if mtype == 3:
        pytest.skip("complex values are not stored")
    coo = W.laplacian_2d(512) if name == "laplace2d_512" else golden_matrices()[name]
    for allow_csr in (True, False):
        want, best = so.block_size_storage(coo.rows, coo.cols, m, n, mtype, allow_csr)
        o = capi.BuildOpts()
        capi.lib.abhsf_build_opts_default(C.byref(o))
        o.matrix_type, o.allow_csr = mtype, int(allow_csr)
        bits = np.zeros(5, np.uint64)
        b = C.c_int32()
        r = np.ascontiguousarray(coo.rows)
        c = np.ascontiguousarray(coo.cols)
        capi.check(capi.lib.abhsf_block_size_storage(r.ctypes.data, c.ctypes.data, coo.nnz, m, n, C.byref(o), None,
                                                     bits.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(b)))
        assert bits.tolist() == want.tolist() and b.value == best


@pytest.mark.parametrize("seed", range(10))
def test_sweep_and_features_match_oracle(gpu, seed):
    import torch
    rows, cols, m, n, name = _small(seed)
    want_bits, want_best = so.block_size_storage(rows, cols, m, n)
    for r, c in ((rows, cols), (torch.from_numpy(rows).cuda(), torch.from_numpy(cols).cuda())):
        bits, best = sel.block_size_storage(r, c, m, n)
        assert bits.tolist() == want_bits.tolist() and best == want_best, name
        f = sel.features(r, c, m, n)
        np.testing.assert_allclose(f, so.features(rows, cols, m, n), **FEAT_TOL, err_msg=name)


def test_features_reject_out_of_range_indices(gpu):
    rows = np.array([0, 5], np.int64)
    cols = np.array([0, 1], np.int64)
    with pytest.raises(capi.IndexOutOfRange):
        sel.features(rows, cols, 5, 5)
    with pytest.raises(capi.IndexOutOfRange):
        sel.block_size_storage(rows, cols, 5, 5)


def _params(seed):
    rng = np.random.default_rng(seed)
    p = (rng.standard_normal(so.P) * 0.3).astype(np.float32)
    p[so.OMEAN:so.OISTD] = rng.standard_normal(so.F) * 0.1
    p[so.OISTD:] = rng.uniform(0.5, 2.0, so.F)
    return p


@pytest.mark.parametrize("batch", [1, 5, 300])
def test_mlp_forward_backward_match_oracle(gpu, batch):
    import torch
    rng = np.random.default_rng(batch)
    p = _params(batch)
    X = rng.standard_normal((batch, so.F)).astype(np.float32)
    T = sel.targets_from_bits(rng.integers(100, 200, (batch, 5)).astype(np.uint64), tau=0.1)
    net = sel.Mlp(p)
    xt, tt = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    probs, act = net.forward(xt, keep=True)
    want_p, (_, _, h1, _, h2) = so.forward(p, X)
    np.testing.assert_allclose(probs.cpu().numpy(), want_p, **PROB_TOL)
    np.testing.assert_allclose(act.cpu().numpy()[:, :64], h1, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(act.cpu().numpy()[:, 64:], h2, rtol=1e-5, atol=1e-5)
    net.g.fill_(123.0)
    net.backward(xt, tt, probs, act)
    g = net.g.cpu().numpy()
    want_g, want_loss = so.backward(p, X, T)
    np.testing.assert_allclose(g[:so.OMEAN], want_g[:so.OMEAN], **GRAD_TOL)
    assert np.all(g[so.OMEAN:] == 123.0)  # the normalisation's entries are left alone
    assert abs(float(net.loss) - want_loss) <= 1e-5 * max(1.0, want_loss)
    # the same gradient again: sums in sample order are reproducible
    net.backward(xt, tt, probs, act)
    assert np.array_equal(net.g.cpu().numpy(), g)


def test_mlp_adam_matches_oracle(gpu):
    import torch
    rng = np.random.default_rng(7)
    p = _params(7)
    net = sel.Mlp(p)
    m = np.zeros(so.P)
    v = np.zeros(so.P)
    want = p.astype(np.float64)
    for step in range(1, 4):
        g = rng.standard_normal(so.P).astype(np.float32)
        net.g.copy_(torch.from_numpy(g))
        net.adam(1e-2)
        want, m, v = so.adam(want, g, m, v, step, 1e-2)
    np.testing.assert_allclose(net.params(), want, rtol=1e-5, atol=1e-6)
    assert np.array_equal(net.params()[so.OMEAN:], p[so.OMEAN:])


def test_training_kernels_reduce_the_loss(gpu):
    import torch
    rng = np.random.default_rng(3)
    X = rng.standard_normal((256, so.F)).astype(np.float32)
    labels = (X[:, 0] > 0).astype(int) + 2 * (X[:, 1] > 0).astype(int)
    T = np.eye(5, dtype=np.float32)[labels]
    net = sel.Mlp(sel.init_params(X, 0))
    xt, tt = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    losses = []
    for _ in range(300):
        probs, act = net.forward(xt, keep=True)
        net.backward(xt, tt, probs, act)
        losses.append(float(net.loss))
        net.adam(3e-3)
    assert losses[-1] < 0.2 * losses[0]
    acc = (sel.choose(net.params(), X) == labels).mean()
    assert acc > 0.95


def test_build_auto_block_size(gpu):
    rows, cols, m, n, name = _small(11)
    vals = np.random.default_rng(0).standard_normal(rows.size)
    _, best = so.block_size_storage(rows, cols, m, n)
    A = AbhsfMatrix.from_elements(rows, cols, vals, m, n, block_size="auto")
    assert A.block_size == best and A.stats()["block_size"] == best
    B = AbhsfMatrix.from_elements(rows, cols, vals, m, n, block_size=best)
    ea, eb = A.export(), B.export()
    for k in ea:
        assert np.array_equal(ea[k], eb[k]), k
    # learned: a model whose output bias always picks 128
    p = sel.untrained_model()
    p[so.OB3:so.OMEAN] = [0, 0, 0, 1, 0]
    L = AbhsfMatrix.from_elements(rows, cols, vals, m, n, block_size="auto", selector="learned", selector_model=p)
    assert L.block_size == 128
    f = sel.features(rows, cols, m, n)
    L2 = AbhsfMatrix.from_elements(rows, cols, vals, m, n, block_size="auto", selector="learned")
    assert L2.block_size == sel.predict(f) in capi.BLOCK_SIZES
    for M in (A, B, L, L2):
        M.release()


def test_learned_selector_beats_a_fixed_block_size(gpu):
    """Held-out matrices (seeds beyond the training range): the shipped model's
    average regret (consistency.cpp:147-173) is below that of always using
    s = 64 and of every other fixed size."""
    import torch
    X, bits = [], []
    for seed in range(5000, 5060):
        r, c, m, n, _ = W.selector_matrix(seed, n_max=1_000_000, nnz_max=4_000_000)
        X.append(sel.features(r, c, m, n))
        bits.append(sel.block_size_storage(r, c, m, n)[0])
        del r, c
    torch.cuda.synchronize()
    X, bits = np.array(X), np.array(bits)
    learned = sel.regret_summary(bits, sel.choose(sel.builtin_model(), X))
    fixed = [sel.regret_summary(bits, np.full(len(X), k)) for k in range(5)]
    assert learned["avg_pct"] < min(f["avg_pct"] for f in fixed), (learned, fixed)
    assert learned["avg_pct"] < 0.5 * fixed[2]["avg_pct"], (learned, fixed[2])


def test_autotune_times_every_size_and_keeps_the_fastest(gpu):
    import torch
    rows, cols, m, n, name = _small(12)
    vals = np.random.default_rng(1).standard_normal(rows.size)
    ms, best, A = sel.autotune(rows, cols, vals, m, n, reps=5, keep=True)
    assert np.all(ms > 0) and best == sel.SIZES[int(np.argmin(ms))] and A.block_size == best
    B = AbhsfMatrix.from_elements(rows, cols, vals, m, n, block_size=best)
    ea, eb = A.export(), B.export()
    for k in ea:
        assert np.array_equal(ea[k], eb[k]), k
    x = torch.from_numpy(np.random.default_rng(2).uniform(-1, 1, n)).cuda()
    ya = torch.zeros(m, dtype=torch.float64, device="cuda")
    yb = ya.clone()
    A.spmv(x, ya)
    B.spmv(x, yb)
    assert torch.equal(ya, yb)
    # device inputs, one candidate
    ms1, best1, _ = sel.autotune(torch.from_numpy(rows).cuda(), torch.from_numpy(cols).cuda(),
                                 torch.from_numpy(vals).cuda(), m, n, candidates=(128,), reps=2)
    assert best1 == 128 and ms1[3] > 0 and np.all(np.delete(ms1, 3) == -1)
    # f32 values: abhsf_spmv_f32 serves every size, so all five are timed
    ms2, best2, _ = sel.autotune(rows, cols, vals, m, n, reps=2, value_type="f32")
    assert np.all(ms2 > 0) and best2 == sel.SIZES[int(np.argmin(ms2))]
    C_ = AbhsfMatrix.from_elements(rows, cols, vals, m, n, block_size="auto", selector="autotune")
    assert C_.block_size in capi.BLOCK_SIZES
    for M in (A, B, C_):
        M.release()


def test_autotune_arguments(gpu):
    rows = np.array([0, 1], np.int64)
    cols = np.array([0, 1], np.int64)
    vals = np.array([1.0, 2.0])
    ms = np.zeros(5, np.float32)
    b = C.c_int32()
    for cand, reps in ((32, 1), (-1, 1), (1, 0)):
        st = capi.lib.abhsf_autotune(rows.ctypes.data, cols.ctypes.data, vals.ctypes.data, 2, 2, 2, None, cand,
                                     reps, None, ms.ctypes.data_as(C.POINTER(C.c_float)), C.byref(b), None)
        assert st == capi.INVALID_VALUE
    # a full 16 x 16 block is a dense tile at size 16: no row slice takes it,
    # the streaming kernel does
    r, c = np.divmod(np.arange(256, dtype=np.int64), 16)
    ms16, best16, _ = sel.autotune(r, c, np.ones(256), 16, 16, candidates=(16,), value_type="bf16")
    assert best16 == 16 and ms16[0] > 0
