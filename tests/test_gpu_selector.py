"""GPU: structure statistics and the MLP selector's CUDA kernels against the
CPU oracle (oracle/selector_ref.py)."""
import numpy as np
import pytest

import oracle
import perf_libs_sparse_b200 as pls
from oracle import selector_ref as R
from perf_libs_sparse_b200 import selector as S
from perf_libs_sparse_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _mats():
    rng = np.random.default_rng(40)
    out = []
    m, n, rp, c, v = W.laplacian_2d(40)
    out.append((m, n, rp, c, v))
    m, n, rp, c, v = W.zipf_rows(6000, seed=41)
    out.append((m, n, rp, c, v))
    rp, c, v = W.random_csr(3000, 5000, 60, rng, empty_frac=0.2)
    out.append((3000, 5000, rp, c, v))
    m, n, rp, c, v = W.stencil_27pt(12, seed=2)
    out.append((m, n, rp, c, v))
    return out


def test_features_match_oracle():
    for m, n, rp, c, v in _mats():
        A = pls.SpMat.csr(m, n, rp, c, v)
        f = S.features(A)
        g = R.features(rp, c, n)
        np.testing.assert_allclose(f, g, rtol=2e-5, atol=2e-6)


def test_mlp_loss_and_gradient_match_cpu_oracle():
    K = len(S.candidates())
    sel = S.Selector(K, seed=3)
    p = sel.get_params()
    rng = np.random.default_rng(5)
    # non-trivial normalisation
    p[-2 * R.NF:-R.NF] = rng.normal(0, 1, R.NF)
    p[-R.NF:] = rng.uniform(0.5, 2.0, R.NF)
    sel.set_params(p)
    X = rng.normal(0, 2, (96, R.NF)).astype(np.float32)
    T = S.soft_targets(rng.uniform(0.1, 2.0, (96, K)))
    loss, g = sel.loss_grad(X, T)
    loss_ref, g_ref = R.mlp_loss_grad(p.astype(np.float64), K, X, T)
    assert abs(loss - loss_ref) <= 1e-5 * max(1.0, abs(loss_ref))
    err = np.abs(g - g_ref).max() / max(np.abs(g_ref).max(), 1e-12)
    assert err <= 1e-4, err


def test_training_lowers_loss_and_learns_a_rule():
    K = len(S.candidates())
    rng = np.random.default_rng(7)
    X = rng.normal(0, 1, (1024, R.NF)).astype(np.float32)
    # the best class is a function of two features
    best = (X[:, 3] > 0).astype(int) * 7 + (X[:, 8] > 0).astype(int) * 3
    times = np.ones((1024, K)) * 2.0
    times[np.arange(1024), best] = 1.0
    T = S.soft_targets(times)
    sel = S.Selector(K, seed=1)
    l0, _ = sel.loss_grad(X, T)
    l1 = sel.train(X, T, epochs=60, batch=128, lr=3e-3, seed=0)
    assert l1 < 0.5 * l0
    _, cls = sel.predict(X)
    assert (cls == best).mean() > 0.9


def test_selector_drives_optimize():
    K = len(S.candidates())
    cands = S.candidates()
    sel = S.Selector(K, seed=2)
    m, n, rp, c, v = W.zipf_rows(20000, seed=9)
    x = W.uniform_vector(n, 10)
    A = pls.SpMat.csr(m, n, rp, c, v)
    f = S.features(A)
    _, cls = sel.predict(f[None, :])
    sel.attach(A)
    A.set_tuner(pls.TUNE_SELECTOR)
    assert A.optimize() == 0
    cfg = A.config()
    kind, C_, sigma, tpr = cands[cls[0]]
    assert cfg["kind"] == (pls.KIND_SELL if kind == pls.KIND_SELL else kind)
    if kind == pls.KIND_SELL:
        assert (cfg["C"], cfg["sigma"]) == (C_, sigma)
    y = A.spmv(x)
    y_ref = oracle.csr_spmv(rp, c, v, x)
    scale = oracle.csr_absdot(rp, c, v, x)
    assert (np.abs(y - y_ref) / np.maximum(np.maximum(np.abs(y_ref), scale), 1e-300)).max() <= 1e-12
