"""CPU: the oracle restatement against the reference's golden vectors and
against the reference library itself (oracle/_ref, when built)."""
import numpy as np
import pytest

import oracle
from tests.conftest import case_names

pytestmark = pytest.mark.filterwarnings("ignore")


def test_spmv_basic_kat(kats):
    k = kats["spmv_basic_d"]
    rp = np.array(k["row_ptr"], np.int32)
    c = np.array(k["col"], np.int32)
    v = np.array(k["vals"], np.float64)
    x = np.array(k["x"], np.float64)
    for mode in (0, 1):
        y = oracle.csr_spmv(rp, c, v, x, alpha=k["alpha"], beta=k["beta"], mode=mode)
        np.testing.assert_allclose(y, k["y"], atol=k["tol"])


def test_bsr_kats(kats):
    k = kats["bsr_row_major"]
    rp = np.array(k["row_ptr"], np.int32)
    c = np.array(k["col"], np.int32)
    v = np.array(k["vals"], np.float64)
    x = np.array(k["x"], np.float64)
    y = oracle.bsr_spmv(rp, c, v, k["bs"], k["layout"], x)
    np.testing.assert_allclose(y, k["y_notrans"], atol=k["tol"])
    crp, cc, cv = oracle.bsr2csr(rp, c, v, k["bs"], k["layout"])
    yt = oracle.csr_spmv_trans(crp, cc, cv, k["n"], x)
    np.testing.assert_allclose(yt, k["y_trans"], atol=k["tol"])

    k = kats["bsr_col_major"]
    rp = np.array(k["row_ptr"], np.int32)
    c = np.array(k["col"], np.int32)
    v = np.array(k["vals"], np.float64)
    crp, cc, cv = oracle.bsr2csr(rp, c, v, k["bs"], k["layout"])
    assert oracle.csr_inf_norm(crp, cv) == k["inf_norm"]
    yt = oracle.csr_spmv_trans(crp, cc, cv, k["n"], np.array(k["x"], float), alpha=k["alpha_trans"])
    np.testing.assert_allclose(yt, k["y_trans_scaled"], atol=k["tol"])


def test_spmm_kats(kats):
    k = kats["matmul_variants_d"]
    rp = np.array(k["row_ptr"], np.int32)
    c = np.array(k["col"], np.int32)
    v = np.array(k["vals"], np.float64)
    A = np.array(k["denseA"]).reshape(4, 4)
    B = np.array(k["denseB"]).reshape(4, 4)
    C0 = np.array(k["c_init"]).reshape(4, 4)
    got = oracle.csr_spmm(rp, c, v, B, 4, alpha=1.0, beta=0.0)
    np.testing.assert_allclose(got, A @ B, atol=k["tol"])
    got = oracle.csr_spmm(rp, c, v, B, 4, Cmat=C0, alpha=k["alpha_beta"], beta=k["beta"])
    np.testing.assert_allclose(got, k["alpha_beta"] * A @ B + C0, atol=k["tol"])


def test_csr2bsr_roundtrip():
    rng = np.random.default_rng(5)
    from perf_libs_sparse_b200 import workloads as W
    for bs in (2, 4, 8):
        for layout in (90, 91):
            m = n = bs * 9
            rp, c, v = W.random_csr(m, n, 10, rng, empty_frac=0.2)
            brp, bc, bv = oracle.csr2bsr(rp, c, v, m, n, bs, layout)
            rp2, c2, v2 = oracle.bsr2csr(brp, bc, bv, bs, layout)
            np.testing.assert_array_equal(rp2, rp)
            np.testing.assert_array_equal(c2, c)
            np.testing.assert_array_equal(v2, v)


def test_port_matches_reference_fixtures(ref_outputs):
    """Restated SELL builder and CSR exec vs the reference library's own
    outputs (committed fixtures made by tests/golden/make_golden.py)."""
    f = ref_outputs
    for name in case_names(f):
        rp, c, v = f[f"{name}/row_ptr"], f[f"{name}/col"], f[f"{name}/vals"]
        m, n = (int(t) for t in f[f"{name}/shape"])
        x, y0 = f[f"{name}/x"], f[f"{name}/y0"]
        y = oracle.csr_spmv(rp, c, v, x, y=y0, alpha=1.5, beta=-0.5, mode=1)
        np.testing.assert_allclose(y, f[f"{name}/y_csr"], rtol=1e-12, atol=1e-12)
        for key in [k[: -len("/info")] for k in f.files if k.startswith(name + "/scs_") and k.endswith("/info")]:
            info = f[key + "/info"]
            C, sigma = int(info[1]), int(info[2])
            s = oracle.scs_build(rp, c, v, n, C, sigma)
            got = [s["nC"], s["C"], s["sigma"], s["col_bytes"], s["n_full_chunks"], s["ntidyup"], s["size"]]
            assert got == [int(t) for t in info], key
            for fld in ("cs", "cl", "col_min", "permd2in", "vals"):
                np.testing.assert_array_equal(s[fld], f[f"{key}/{fld}"], err_msg=f"{key}/{fld}")
            np.testing.assert_array_equal(s["offsets"], f[f"{key}/offsets"].astype(np.int64))


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_port_matches_reference_live():
    """Live cross-check on fresh random cases, including SELL exec (C <= 16,
    the sizes the reference executes)."""
    from perf_libs_sparse_b200 import workloads as W
    rng = np.random.default_rng(99)
    for t in range(25):
        m = int(rng.integers(1, 400))
        n = int(rng.integers(1, 900))
        rp, c, v = W.random_csr(m, n, min(n, 40), rng, base=int(t % 2))
        for C in (2, 8, 16, 32):
            for sigma in (0, C, 4 * C):
                a = oracle.ref_scs_build(rp, c, v, n, C, sigma)
                b = oracle.scs_build(rp, c, v, n, C, sigma)
                for k in ("cs", "cl", "col_min", "permd2in", "in2permd", "vals", "offsets"):
                    np.testing.assert_array_equal(a[k], b[k])
                assert (a["col_bytes"], a["n_full_chunks"], a["ntidyup"]) == (
                    b["col_bytes"], b["n_full_chunks"], b["ntidyup"])
                x = rng.uniform(-1, 1, n)
                yp = oracle.scs_spmv(b, x, alpha=1.0)
                assert np.all(np.isfinite(yp))


def test_mlp_oracle_gradient_finite_differences():
    """The CPU restatement of the selector MLP is itself checked against
    central finite differences (FP64)."""
    from oracle import selector_ref as R

    K = 7
    rng = np.random.default_rng(0)
    P = R.H * R.NF + R.H + R.H * R.H + R.H + K * R.H + K
    p = np.concatenate([rng.normal(0, 0.3, P), rng.normal(0, 1, R.NF), rng.uniform(0.5, 2, R.NF)])
    X = rng.normal(0, 1, (10, R.NF))
    T = rng.dirichlet(np.ones(K), 10)
    loss, g = R.mlp_loss_grad(p, K, X, T)
    for i in rng.choice(P, 40, replace=False):
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (R.mlp_loss_grad(p + e, K, X, T)[0] - R.mlp_loss_grad(p - e, K, X, T)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), i


def test_scs_spmv_equals_csr():
    from perf_libs_sparse_b200 import workloads as W
    rng = np.random.default_rng(3)
    rp, c, v = W.random_csr(500, 700, 50, rng)
    x = rng.uniform(-1, 1, 700)
    y_ref = oracle.csr_spmv(rp, c, v, x)
    for C in (8, 32):
        for sigma in (0, 64 * C // 8):
            s = oracle.scs_build(rp, c, v, 700, C, sigma)
            y = oracle.scs_spmv(s, x)
            np.testing.assert_allclose(y, y_ref, rtol=1e-12, atol=1e-12)


def _random_coo(rng, m, n, nnz, unique):
    r = rng.integers(0, m, nnz).astype(np.int32)
    c = rng.integers(0, n, nnz).astype(np.int32)
    v = rng.normal(size=nnz)
    if unique:
        _, ui = np.unique(r.astype(np.int64) * n + c, return_index=True)
        ui = np.sort(ui)
        r, c, v = r[ui], c[ui], v[ui]
    return r, c, v


def _csc_of(m, n, r, c, v):
    order = np.lexsort((r, c))  # by column, then row
    cp = np.zeros(n + 1, np.int32)
    np.add.at(cp, c + 1, 1)
    return r[order].astype(np.int32), np.cumsum(cp).astype(np.int32), v[order]


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_coo_csc_restatement_matches_reference():
    """coo2csr / csc2csr restated in the oracle against the reference
    library's own conversion (its export_csr converts COO / CSC handles to
    CSR): bit-exact for distinct positions; with duplicates the structure is
    exact and the values agree as a multiset (the reference's std::sort
    leaves the order of equal positions unspecified)."""
    rng = np.random.default_rng(5)
    for t in range(20):
        m, n = int(rng.integers(1, 300)), int(rng.integers(1, 300))
        nnz = int(rng.integers(0, 3 * (m + n)))
        r, c, v = _random_coo(rng, m, n, nnz, unique=True)
        ours = oracle.coo2csr(m, n, r, c, v)
        theirs = oracle.RefMatrix.coo(m, n, r, c, v).export_csr(m)
        for a, b in zip(ours, theirs):
            np.testing.assert_array_equal(a, b)
        ri, cp, cv = _csc_of(m, n, r, c, v)
        for base in (0, 1):
            ours = oracle.csc2csr(m, n, ri + base, cp + base, cv)
            theirs = oracle.RefMatrix.csc(m, n, ri + base, cp + base, cv).export_csr(m, index_base=base)
            for a, b in zip(ours, theirs):
                np.testing.assert_array_equal(a, b)
        r, c, v = _random_coo(rng, m, n, nnz, unique=False)
        o_rp, o_c, o_v = oracle.coo2csr(m, n, r, c, v)
        t_rp, t_c, t_v = oracle.RefMatrix.coo(m, n, r, c, v).export_csr(m)
        np.testing.assert_array_equal(o_rp, t_rp)
        np.testing.assert_array_equal(o_c, t_c)
        np.testing.assert_array_equal(np.sort(o_v), np.sort(t_v))


def test_spmm_port_matches_reference_fixtures(ref_spmm):
    """The restated SpMM (oracle.csr_spmm, the blocked row-wise loop of
    src/compressed_sparse_rows.cpp:1699-1764) against the reference's own
    perflibs_spmm_exec_d outputs (tests/golden/ref_spmm.npz): CSR with index
    base 0 and 1, BSR bs 4 and 8 in both block layouts through its CSR view,
    k in {4, 8, 32, 128} (k = 4 is the reference's repeated-SpMV route), with
    and without beta. Per-row scaled error <= 1e-12: summation order is the
    only freedom."""
    from tests.conftest import spmm_case_csr, spmm_row_err

    f = ref_spmm
    names = sorted({k.split("/")[0] for k in f.files})
    assert len(names) == 7
    for name in names:
        rp, col, vals = spmm_case_csr(f, name)
        B, C0 = f[f"{name}/B"], f[f"{name}/C0"]
        for k in (int(t) for t in f[f"{name}/ks"]):
            Bk = np.ascontiguousarray(B[:, :k])
            got = oracle.csr_spmm(rp, col, vals, Bk, k, alpha=1.5)
            assert spmm_row_err(got, f[f"{name}/C_k{k}"], rp, col, vals, Bk, 1.5) <= 1e-12, (name, k)
            if k >= 8:  # the blocked loop: the same order as the reference, bit for bit
                np.testing.assert_array_equal(got, f[f"{name}/C_k{k}"], err_msg=f"{name} k={k}")
            if f"{name}/Cb_k{k}" in f.files:
                C0k = np.ascontiguousarray(C0[:, :k])
                got = oracle.csr_spmm(rp, col, vals, Bk, k, Cmat=C0k, alpha=0.75, beta=-0.5)
                assert spmm_row_err(got, f[f"{name}/Cb_k{k}"], rp, col, vals, Bk, 0.75, -0.5, C0k) <= 1e-12, (name, k)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_spmm_port_matches_reference_live():
    """Fresh random CSR SpMMs, the port against the reference library run
    here, k across the repeated-SpMV threshold."""
    from perf_libs_sparse_b200 import workloads as W
    from tests.conftest import spmm_row_err

    rng = np.random.default_rng(77)
    for t in range(12):
        m, n = int(rng.integers(1, 200)), int(rng.integers(1, 200))
        rp, c, v = W.random_csr(m, n, min(n, 30), rng)
        k = int(rng.choice([1, 3, 4, 5, 8, 17, 64]))
        B = rng.uniform(-1, 1, (n, k))
        A = oracle.RefMatrix.csr(m, n, rp, c, v)
        theirs = A.spmm(m, B, alpha=-1.25)
        A.destroy()
        ours = oracle.csr_spmm(rp, c, v, B, k, alpha=-1.25)
        assert spmm_row_err(ours, theirs, rp, c, v, B, -1.25) <= 1e-12, (m, n, k)
