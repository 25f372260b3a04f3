"""GPU: every SpMV kernel configuration the tuner can pick (CSR threads per
row, CSR long-row split, SELL C x sigma), forced one at a time, on edge
matrices, against the oracle row by row (FP64, <= 1e-12 scaled)."""
import numpy as np
import pytest

import oracle
import perf_libs_sparse_b200 as pls
from perf_libs_sparse_b200 import selector as S

pytestmark = pytest.mark.gpu


def _csr_from_lengths(lens, n, rng):
    rp = np.zeros(len(lens) + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    cols = [np.sort(rng.choice(n, size=int(l), replace=False)) for l in lens]
    col = np.concatenate(cols).astype(np.int32) if len(cols) else np.zeros(0, np.int32)
    return rp, col, rng.normal(size=int(rp[-1]))


def _matrices():
    rng = np.random.default_rng(17)
    out = {}
    out["one_row"] = (1, 50) + _csr_from_lengths([37], 50, rng)
    out["one_col"] = (40, 1) + _csr_from_lengths(rng.integers(0, 2, 40), 1, rng)
    lens = rng.integers(0, 9, 1003)  # ragged last chunk for C = 8/16/32
    out["ragged"] = (1003, 700) + _csr_from_lengths(lens, 700, rng)
    lens = np.zeros(3000, int)
    lens[1234] = 20000  # one very long row among empty ones
    lens[rng.choice(3000, 200, replace=False)] = rng.integers(1, 5, 200)
    out["one_long_row"] = (3000, 40000) + _csr_from_lengths(lens, 40000, rng)
    lens = np.minimum(rng.zipf(1.7, 5000), 3000)
    out["power_law"] = (5000, 5000) + _csr_from_lengths(lens, 5000, rng)
    return out


MATS = _matrices()


@pytest.fixture(scope="module")
def candidates():
    return S.candidates()


@pytest.mark.parametrize("name", sorted(MATS))
def test_every_config_on_edge_matrices(name, candidates):
    m, n, rp, col, val = MATS[name]
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, n)
    y0 = rng.uniform(-1, 1, m)
    for alpha, beta in [(1.0, 0.0), (-2.5, 1.0), (0.75, -0.5)]:
        ref = oracle.csr_spmv(rp, col, val, x, y=y0.copy(), alpha=alpha, beta=beta)
        scale = abs(alpha) * oracle.csr_absdot(rp, col, val, x) + abs(beta) * np.abs(y0)
        den = np.maximum(np.abs(ref), scale)
        den[den == 0] = 1
        for kind, C_, sigma, tpr in candidates:
            A = pls.SpMat.csr(m, n, rp, col, val)
            assert A.force_config(int(kind), int(C_), int(sigma), int(tpr)) == 0
            assert A.optimize() == 0
            y = A.spmv(x, y0.copy(), alpha=alpha, beta=beta)
            err = (np.abs(y - ref) / den).max() if m else 0.0
            assert err <= 1e-12, (name, kind, C_, sigma, tpr, alpha, beta, err)


def test_one_based_input_every_family(candidates):
    m, n, rp, col, val = MATS["ragged"]
    x = np.random.default_rng(5).uniform(-1, 1, n)
    ref = oracle.csr_spmv(rp, col, val, x)
    for kind, C_, sigma, tpr in candidates[::4]:
        A = pls.SpMat.csr(m, n, rp + 1, col + 1, val)
        A.force_config(int(kind), int(C_), int(sigma), int(tpr))
        assert A.optimize() == 0
        np.testing.assert_allclose(A.spmv(x), ref, rtol=1e-12, atol=1e-12)
        _, _, erp, ecol, evals = A.export_csr(index_base=1)
        # export keeps the base asked for (zeros dropped after SELL)
        assert erp[0] == 1 and (len(ecol) == 0 or ecol.min() >= 1)


def test_inf_and_nan_propagate_like_the_reference(candidates):
    """Inf / NaN in x: CSR kernels follow the CSR oracle; SELL kernels follow
    the restated reference SELL kernel, whose padding slots (value 0,
    offset 0) also multiply x at the chunk's smallest column
    (src/sell_c_sigma.cpp:727-775), so 0 * Inf makes a NaN there exactly as
    in the reference."""
    m, n, rp, col, val = MATS["ragged"]
    x = np.random.default_rng(6).uniform(-1, 1, n)
    x[col[5]] = np.inf
    x[col[100]] = np.nan
    ref_csr = oracle.csr_spmv(rp, col, val, x)
    for kind, C_, sigma, tpr in candidates:
        if int(kind) == pls.KIND_SELL:
            lay = oracle.scs_build(rp, col, val, n, int(C_), int(sigma))
            ref = oracle.scs_spmv(lay, x)
        else:
            ref = ref_csr
        A = pls.SpMat.csr(m, n, rp, col, val)
        A.force_config(int(kind), int(C_), int(sigma), int(tpr))
        assert A.optimize() == 0
        y = A.spmv(x)
        np.testing.assert_array_equal(np.isnan(y), np.isnan(ref), err_msg=str((kind, C_, sigma, tpr)))
        np.testing.assert_array_equal(np.isinf(y), np.isinf(ref), err_msg=str((kind, C_, sigma, tpr)))
        fin = np.isfinite(ref)
        np.testing.assert_allclose(y[fin], ref[fin], rtol=1e-12, atol=1e-12)
