"""GPU: bit-exact layout conversions (CSR -> SELL-C-sigma, CSR -> BSR),
export, and norms, against the oracle."""
import numpy as np
import pytest

import oracle
import perf_libs_sparse_b200 as pls
from perf_libs_sparse_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_sell_layout_random_bit_exact():
    rng = np.random.default_rng(17)
    for t in range(12):
        m = int(rng.integers(1, 3000))
        n = int(rng.integers(1, 5000))
        base = t % 2
        rp, c, v = W.random_csr(m, n, min(n, 90), rng, base=base, empty_frac=0.25)
        A = pls.SpMat.csr(m, n, rp, c, v)
        for C in (8, 16, 32):
            for sigma in (0, C, 8 * C, 16384 // C * C):
                assert A.build_sell(C, sigma) == 0
                g = A.export_sell()
                o = oracle.scs_build(rp, c, v, n, C, sigma)
                for k in ("nC", "size", "col_bytes", "n_full_chunks", "ntidyup"):
                    assert g[k] == o[k], (k, m, n, C, sigma)
                for k in ("cs", "cl", "col_min", "permd2in", "in2permd", "vals", "offsets"):
                    np.testing.assert_array_equal(g[k], o[k], err_msg=f"{k} m={m} n={n} C={C} s={sigma}")


def test_sell_layout_full_size_zipf_properties():
    """C2-sized matrix: the device layout equals the oracle layout on a
    seeded 1M-row power-law matrix (sigma = 8192), and every row's entries
    appear exactly once."""
    m, n, rp, c, v = W.zipf_rows(1 << 20, seed=1)
    A = pls.SpMat.csr(m, n, rp, c, v)
    assert A.build_sell(32, 8192) == 0
    g = A.export_sell()
    o = oracle.scs_build(rp, c, v, n, 32, 8192)
    for k in ("cs", "cl", "col_min", "permd2in", "vals", "offsets"):
        np.testing.assert_array_equal(g[k], o[k], err_msg=k)
    assert np.count_nonzero(g["vals"]) == np.count_nonzero(v)
    assert abs(oracle.scs_beta(o, int(rp[-1])) - int(rp[-1]) / g["size"]) < 1e-15 or g["ntidyup"] > 0


def test_csr_to_bsr_bit_exact():
    rng = np.random.default_rng(23)
    for bs in (1, 2, 4, 8):
        for layout in (pls.ROW_MAJOR, pls.COL_MAJOR):
            m, n = bs * 37, bs * 29
            base = bs % 2
            rp, c, v = W.random_csr(m, n, 15, rng, base=base)
            A = pls.SpMat.csr(m, n, rp, c, v)
            B = A.to_bsr(bs, layout)
            gbs, grp, gc, gv = B.export_bsr()
            orp, oc, ov = oracle.csr2bsr(rp, c, v, m, n, bs, layout)
            assert gbs == bs
            np.testing.assert_array_equal(grp, orp)
            np.testing.assert_array_equal(gc, oc)
            np.testing.assert_array_equal(gv, ov)
            # round trip through the reference's bsr2csr semantics
            rp2, c2, v2 = oracle.bsr2csr(orp, oc, ov, bs, layout)
            np.testing.assert_array_equal(rp2, rp)
            np.testing.assert_array_equal(c2, c)
            np.testing.assert_array_equal(v2, v)
            # and the device's own export of the BSR handle
            _, _, rp3, c3, v3 = B.export_csr(base)
            np.testing.assert_array_equal(rp3, rp)
            np.testing.assert_array_equal(c3, c)
            np.testing.assert_array_equal(v3, v)


def test_export_after_sell_drops_explicit_zeros():
    rp = np.array([0, 3, 5, 6], np.int32)
    c = np.array([0, 1, 2, 0, 2, 1], np.int32)
    v = np.array([1.0, 0.0, 2.0, 3.0, 0.0, 4.0])
    A = pls.SpMat.csr(3, 3, rp, c, v)
    _, _, rp1, c1, v1 = A.export_csr(0)
    np.testing.assert_array_equal(v1, v)
    A.force_config(pls.KIND_SELL, 8, 0, 0)
    assert A.optimize() == 0
    _, _, rp2, c2, v2 = A.export_csr(1)
    np.testing.assert_array_equal(rp2, [1, 3, 4, 5])
    np.testing.assert_array_equal(c2, [1, 3, 1, 2])
    np.testing.assert_array_equal(v2, [1.0, 2.0, 3.0, 4.0])


def test_norms():
    rng = np.random.default_rng(31)
    rp, c, v = W.random_csr(700, 400, 40, rng)
    A = pls.SpMat.csr(700, 400, rp, c, v)
    assert A.norm(pls.NORM_INF) == pytest.approx(oracle.csr_inf_norm(rp, v), rel=1e-14)
    assert A.norm(pls.NORM_FRB) == pytest.approx(np.sqrt((v ** 2).sum()), rel=1e-13)
    v2 = v.copy()
    v2[5] = np.nan
    B = pls.SpMat.csr(700, 400, rp, c, v2)
    assert np.isnan(B.norm(pls.NORM_INF))
    D = pls.SpMat.dense(pls.COL_MAJOR, 2, 2, 2, np.array([1.0, -3.0, 2.0, 4.0]))
    assert D.norm(pls.NORM_INF) == 7.0


def test_coo_input_matches_oracle():
    """COO creation (device radix sort by (row, column), duplicates kept in
    input order) gives exactly the oracle's CSR; SpMV on it matches."""
    rng = np.random.default_rng(21)
    for m, n, nnz in [(1, 1, 0), (7, 5, 30), (500, 300, 4000), (3000, 2000, 60000)]:
        r = rng.integers(0, m, nnz).astype(np.int32)
        c = rng.integers(0, n, nnz).astype(np.int32)
        v = rng.normal(size=nnz)
        A = pls.SpMat.coo(m, n, r, c, v)
        mm, nn, rp, cc, vv = A.export_csr()
        assert (mm, nn) == (m, n)
        o_rp, o_c, o_v = oracle.coo2csr(m, n, r, c, v)
        np.testing.assert_array_equal(rp, o_rp)
        np.testing.assert_array_equal(cc, o_c)
        np.testing.assert_array_equal(vv, o_v)
        x = rng.uniform(-1, 1, n)
        y = A.spmv(x)
        ref = oracle.csr_spmv(o_rp, o_c, o_v, x)
        sc = oracle.csr_absdot(o_rp, o_c, o_v, x)
        den = np.maximum(np.abs(ref), sc)
        den[den == 0] = 1
        assert (np.abs(y - ref) / den).max() <= 1e-12


def test_csc_input_matches_oracle():
    rng = np.random.default_rng(22)
    for m, n, ml, base in [(40, 60, 5, 0), (800, 500, 20, 1)]:
        rp, c, v = W.random_csr(n, m, ml, rng)  # CSR of A^T = CSC of A
        A = pls.SpMat.csc(m, n, c + base, rp + base, v)
        got = A.export_csr()[2:]
        o_rp, o_c, o_v = oracle.csc2csr(m, n, c, rp, v)
        for a, b in zip(got, (o_rp, o_c, o_v)):
            np.testing.assert_array_equal(a, b)


def test_bad_indices_rejected_before_any_kernel():
    """Indices out of range are input errors (argument position as the
    error code), checked on the device before any kernel indexes with them."""
    rp = np.array([0, 2, 3], np.int32)
    v = np.ones(3)
    A = pls.SpMat.csr(2, 4, rp, np.array([0, 4, 1], np.int32), v, check=False)
    assert A.status == pls.STATUS_INPUT_PARAMETER_ERROR and A.error_code() == 5
    A = pls.SpMat.csr(2, 4, np.array([0, 3, 2], np.int32), np.array([0, 1, 1], np.int32), v,
                      check=False)
    assert A.status == pls.STATUS_INPUT_PARAMETER_ERROR and A.error_code() == 4
    A = pls.SpMat.coo(3, 3, np.array([0, 3], np.int32), np.array([1, 1], np.int32), np.ones(2),
                      check=False)
    assert A.status == pls.STATUS_INPUT_PARAMETER_ERROR and A.error_code() == 5
    A = pls.SpMat.coo(3, 3, np.array([0, 1], np.int32), np.array([-1, 1], np.int32), np.ones(2),
                      check=False)
    assert A.status == pls.STATUS_INPUT_PARAMETER_ERROR and A.error_code() == 6
    A = pls.SpMat.csc(3, 2, np.array([0, 1], np.int32), np.array([2, 1, 2], np.int32),
                      np.ones(2), check=False)
    assert A.status == pls.STATUS_INPUT_PARAMETER_ERROR and A.error_code() == 4
    A = pls.SpMat.csc(3, 2, np.array([0, 5], np.int32), np.array([0, 1, 2], np.int32),
                      np.ones(2), check=False)
    assert A.status == pls.STATUS_INPUT_PARAMETER_ERROR and A.error_code() == 4
