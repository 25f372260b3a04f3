"""GPU parity: sparse x dense SpMM through the C-ABI (drop-in create / hint /
optimize / exec / export flow), against the reference's golden vectors and
the oracle. FP64 tolerance 1e-12 (scaled per element as for SpMV)."""
import numpy as np
import pytest

import oracle
import perf_libs_sparse_b200 as pls
from perf_libs_sparse_b200 import workloads as W
from tests.conftest import rel_err_rows

pytestmark = pytest.mark.gpu


def spmm_ref(rp, c, v, B, alpha, beta, C0):
    return oracle.csr_spmm(rp, c, v, np.ascontiguousarray(B), B.shape[1], Cmat=C0, alpha=alpha, beta=beta)


def scaled_err(got, ref, rp, c, v, B, alpha, beta, C0):
    absA = oracle.csr_spmm(rp, c, np.abs(v), np.abs(np.ascontiguousarray(B)), B.shape[1])
    sc = abs(alpha) * absA
    if C0 is not None and beta != 0:
        sc = sc + abs(beta) * np.abs(C0)
    den = np.maximum(np.abs(ref), sc)
    den[den == 0] = 1
    return (np.abs(got - ref) / den).max()


def dense_scaled_err(got, ref, scale):
    """Elementwise |got - ref| / max(|ref|, scale): the per-element form of
    the scaled metric, for products checked against numpy."""
    den = np.maximum(np.abs(ref), scale)
    den = np.where(den == 0, 1.0, den)
    return float((np.abs(got - ref) / den).max())


def test_kat_matmul_variants(kats):
    k = kats["matmul_variants_d"]
    rp, c, v = np.array(k["row_ptr"]), np.array(k["col"]), np.array(k["vals"])
    Ad = np.array(k["denseA"]).reshape(4, 4)
    Bd = np.array(k["denseB"]).reshape(4, 4)
    A = pls.SpMat.csr(4, 4, rp, c, v)
    B = pls.SpMat.dense(pls.ROW_MAJOR, 4, 4, 4, Bd.reshape(-1))
    opt_null = pls.SpMat.null(4, 4)
    assert pls.spmm_optimize(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, pls.SCALAR_ANY, A, B,
                             pls.SCALAR_ANY, opt_null) == 0
    for ta in (pls.OPERATION_NOTRANS, pls.OPERATION_TRANS):
        for tb in (pls.OPERATION_NOTRANS, pls.OPERATION_TRANS):
            Cm = pls.SpMat.null(4, 4)
            alpha = k["alpha_notrans"] if ta == pls.OPERATION_NOTRANS else k["alpha_trans"]
            assert pls.spmm_exec(ta, tb, alpha, A, B, 0.0, Cm) == 0
            opA = Ad if ta == pls.OPERATION_NOTRANS else Ad.T
            opB = Bd if tb == pls.OPERATION_NOTRANS else Bd.T
            np.testing.assert_allclose(Cm.export_dense(pls.ROW_MAJOR), alpha * opA @ opB, atol=k["tol"])
    C0 = np.array(k["c_init"]).reshape(4, 4)
    Cd = pls.SpMat.dense(pls.ROW_MAJOR, 4, 4, 4, C0.reshape(-1))
    assert pls.spmm_exec(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, k["alpha_beta"], A, B, k["beta"], Cd) == 0
    np.testing.assert_allclose(Cd.export_dense(), k["alpha_beta"] * Ad @ Bd + k["beta"] * C0, atol=k["tol"])
    # column-major B and C
    Bc = pls.SpMat.dense(pls.COL_MAJOR, 4, 4, 4, Bd.T.reshape(-1))
    Cc = pls.SpMat.dense(pls.COL_MAJOR, 4, 4, 4, C0.T.reshape(-1))
    assert pls.spmm_exec(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, k["alpha_beta"], A, Bc, k["beta"], Cc) == 0
    np.testing.assert_allclose(Cc.export_dense(pls.ROW_MAJOR), k["alpha_beta"] * Ad @ Bd + C0, atol=k["tol"])
    np.testing.assert_allclose(Cc.export_dense(pls.COL_MAJOR), k["alpha_beta"] * Ad @ Bd + C0, atol=k["tol"])


def _dense_of(m, n, rp, c, v):
    D = np.zeros((m, n))
    for i in range(m):
        for p in range(rp[i], rp[i + 1]):
            D[i, c[p]] += v[p]
    return D


def test_kat_matmul_dispatch_paths(kats):
    """test/matmul_dispatch_paths_d.c: dense x dense (the reference's
    cblas_dgemm path), dense x sparse, identity x sparse and sparse x
    identity, with the file's own data and expected values."""
    k = kats["matmul_dispatch_paths_d"]
    NT = pls.OPERATION_NOTRANS
    g = k["gemm"]
    A4, B4, C04 = (np.array(g[n]).reshape(4, 4) for n in ("A", "B", "C0"))
    A = pls.SpMat.dense(pls.ROW_MAJOR, 4, 4, 4, np.array(g["A"]))
    B = pls.SpMat.dense(pls.ROW_MAJOR, 4, 4, 4, np.array(g["B"]))
    Cm = pls.SpMat.dense(pls.ROW_MAJOR, 4, 4, 4, np.array(g["C0"]))
    assert pls.spmm_exec(NT, NT, g["alpha"], A, B, g["beta"], Cm) == 0
    np.testing.assert_allclose(Cm.export_dense(), g["alpha"] * A4 @ B4 + g["beta"] * C04,
                               atol=k["tol"])
    d = k["dense_sparse"]
    rp, c, v = np.array(d["row_ptr"]), np.array(d["col"]), np.array(d["vals"])
    Bs = pls.SpMat.csr(4, 4, rp, c, v)
    Ad = pls.SpMat.dense(pls.ROW_MAJOR, 4, 4, 4, np.array(d["A"]))
    Cm = pls.SpMat.null(4, 4)
    assert pls.spmm_exec(NT, NT, 1.0, Ad, Bs, 0.0, Cm) == 0
    Bd = _dense_of(4, 4, rp, c, v)
    np.testing.assert_allclose(Cm.export_dense(), np.array(d["A"]).reshape(4, 4) @ Bd,
                               atol=k["tol"])
    Cm = pls.SpMat.null(4, 4)
    assert pls.spmm_exec(NT, NT, k["identity_left_alpha"], pls.SpMat.identity(4), Bs, 0.0, Cm) == 0
    np.testing.assert_allclose(Cm.export_dense(), k["identity_left_alpha"] * Bd, atol=k["tol"])
    r = k["identity_right"]
    X = pls.SpMat.csr(4, 4, np.array(r["row_ptr"]), np.array(r["col"]), np.array(r["vals"]))
    Cm = pls.SpMat.null(4, 4)
    assert pls.spmm_exec(NT, NT, r["alpha"], X, pls.SpMat.identity(4), 0.0, Cm) == 0
    np.testing.assert_allclose(Cm.export_dense().reshape(-1), r["expected"], atol=k["tol"])


@pytest.mark.parametrize("ta", [pls.OPERATION_NOTRANS, pls.OPERATION_TRANS])
@pytest.mark.parametrize("tb", [pls.OPERATION_NOTRANS, pls.OPERATION_TRANS])
def test_identity_and_dense_products_vs_numpy(ta, tb):
    """Identity factors and dense x dense beyond the reference's cases:
    transposes, rectangular factors, a column-major C, beta != 0 (C = alpha
    op(A) op(B) + beta C), BSR and CSR operands, and I x I."""
    rng = np.random.default_rng(5)
    T = lambda M, t: M.T if t != pls.OPERATION_NOTRANS else M  # noqa: E731
    m, kk, n = 6, 4, 5
    Ad = rng.uniform(-1, 1, (m, kk) if ta == pls.OPERATION_NOTRANS else (kk, m))
    Bd = rng.uniform(-1, 1, (kk, n) if tb == pls.OPERATION_NOTRANS else (n, kk))
    C0 = rng.uniform(-1, 1, (m, n))
    A = pls.SpMat.dense(pls.COL_MAJOR, Ad.shape[0], Ad.shape[1], Ad.shape[0], Ad.T.reshape(-1))
    B = pls.SpMat.dense(pls.ROW_MAJOR, Bd.shape[0], Bd.shape[1], Bd.shape[1], Bd.reshape(-1))
    Cm = pls.SpMat.dense(pls.COL_MAJOR, m, n, m, C0.T.reshape(-1))
    assert pls.spmm_exec(ta, tb, 0.75, A, B, -0.5, Cm) == 0
    ref = 0.75 * T(Ad, ta) @ T(Bd, tb) - 0.5 * C0
    scale = 0.75 * np.abs(T(Ad, ta)) @ np.abs(T(Bd, tb)) + 0.5 * np.abs(C0)
    assert dense_scaled_err(Cm.export_dense(), ref, scale) <= 1e-12
    # identity x sparse (CSR, then BSR) and sparse x identity, beta != 0
    rp, c, v = W.random_csr(6, 6, 4, rng)
    S = _dense_of(6, 6, rp, c, v)
    C1 = rng.uniform(-1, 1, (6, 6))
    for Sm in (pls.SpMat.csr(6, 6, rp, c, v),
               pls.SpMat.bsr(pls.ROW_MAJOR, 6, 6, 2, *oracle.csr2bsr(rp, c, v, 6, 6, 2, pls.ROW_MAJOR))):
        Cm = pls.SpMat.dense(pls.ROW_MAJOR, 6, 6, 6, C1.reshape(-1))
        assert pls.spmm_exec(ta, tb, 1.25, pls.SpMat.identity(6), Sm, 0.5, Cm) == 0
        assert dense_scaled_err(Cm.export_dense(), 1.25 * T(S, tb) + 0.5 * C1,
                                1.25 * np.abs(T(S, tb)) + 0.5 * np.abs(C1)) <= 1e-12
        Cm = pls.SpMat.dense(pls.ROW_MAJOR, 6, 6, 6, C1.reshape(-1))
        assert pls.spmm_exec(ta, tb, -2.0, Sm, pls.SpMat.identity(6), 0.0, Cm) == 0
        assert dense_scaled_err(Cm.export_dense(), -2.0 * T(S, ta), 2.0 * np.abs(T(S, ta))) <= 1e-12
    Cm = pls.SpMat.dense(pls.ROW_MAJOR, 6, 6, 6, C1.reshape(-1))
    assert pls.spmm_exec(ta, tb, 3.0, pls.SpMat.identity(6), pls.SpMat.identity(6), 1.0, Cm) == 0
    assert dense_scaled_err(Cm.export_dense(), 3.0 * np.eye(6) + C1, 3.0 * np.eye(6) + np.abs(C1)) <= 1e-12


def test_kat_matrix_kernel_ops(kats):
    k = kats["matrix_kernel_ops_spmm"]
    rp, c, v = np.array(k["row_ptr"]), np.array(k["col"]), np.array(k["vals"])
    Bd = np.array(k["denseB"]).reshape(4, 4)
    Ad = np.zeros((4, 4))
    for i in range(4):
        for p in range(rp[i], rp[i + 1]):
            Ad[i, c[p]] = v[p]
    A = pls.SpMat.csr(4, 4, rp, c, v)
    B = pls.SpMat.dense(pls.ROW_MAJOR, 4, 4, 4, Bd.reshape(-1))
    Cm = pls.SpMat.null(4, 4)
    assert pls.spmm_optimize(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, pls.SCALAR_ANY, A, B,
                             pls.SCALAR_ZERO, Cm) == 0
    assert pls.spmm_exec(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, 1.0, A, B, 0.0, Cm) == 0
    np.testing.assert_allclose(Cm.export_dense(), Ad @ Bd, atol=k["tol"])


@pytest.mark.parametrize("k", [1, 3, 5, 8, 13, 32, 128, 300])
def test_random_spmm_vs_oracle(k):
    rng = np.random.default_rng(k)
    for m, n, ml, base in [(200, 150, 20, 0), (1500, 1000, 40, 1)]:
        rp, c, v = W.random_csr(m, n, ml, rng, base=base)
        Bd = rng.uniform(-1, 1, (n, k))
        C0 = rng.uniform(-1, 1, (m, k))
        rp0, c0 = rp - base, c - base
        for alpha, beta in [(1.0, 0.0), (1.5, 1.0), (-0.5, 0.25)]:
            A = pls.SpMat.csr(m, n, rp, c, v)
            B = pls.SpMat.dense(pls.ROW_MAJOR, n, k, k, Bd.reshape(-1))
            Cm = pls.SpMat.dense(pls.ROW_MAJOR, m, k, k, C0.reshape(-1)) if beta != 0 else pls.SpMat.null(m, k)
            assert pls.spmm_optimize(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, pls.SCALAR_ANY, A, B,
                                     pls.SCALAR_ANY if beta else pls.SCALAR_ZERO, Cm) == 0
            assert pls.spmm_exec(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, alpha, A, B, beta, Cm) == 0
            got = Cm.export_dense()
            ref = spmm_ref(rp0, c0, v, Bd, alpha, beta, C0 if beta else None)
            assert scaled_err(got, ref, rp0, c0, v, Bd, alpha, beta, C0) <= 1e-12, (m, k, alpha, beta)


@pytest.mark.parametrize("k", [7, 64, 200])
def test_random_spmm_fp32_vs_oracle(k):
    """FP32 API: 16-byte vectors (k = 64, 200 with several column tiles) and
    scalar columns (k = 7); FP32 accumulation, scaled error <= 1e-5."""
    rng = np.random.default_rng(100 + k)
    m, n = 900, 700
    rp, c, v = W.random_csr(m, n, 50, rng)
    Bd = rng.uniform(-1, 1, (n, k)).astype(np.float32)
    C0 = rng.uniform(-1, 1, (m, k)).astype(np.float32)
    A = pls.SpMat.csr(m, n, rp, c, v.astype(np.float32))
    B = pls.SpMat.dense(pls.ROW_MAJOR, n, k, k, Bd.reshape(-1))
    Cm = pls.SpMat.dense(pls.ROW_MAJOR, m, k, k, C0.reshape(-1))
    assert pls.spmm_exec(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, 1.25, A, B, 0.5, Cm) == 0
    got = Cm.export_dense().astype(np.float64)
    v32 = v.astype(np.float32).astype(np.float64)
    ref = spmm_ref(rp, c, v32, Bd.astype(np.float64), 1.25, 0.5, C0.astype(np.float64))
    assert scaled_err(got, ref, rp, c, v32, Bd.astype(np.float64), 1.25, 0.5, C0.astype(np.float64)) <= 1e-5


def test_repeated_exec_with_beta_zero_overwrites():
    rng = np.random.default_rng(2)
    rp, c, v = W.random_csr(300, 300, 10, rng)
    Bd = rng.uniform(-1, 1, (300, 16))
    A = pls.SpMat.csr(300, 300, rp, c, v)
    B = pls.SpMat.dense(pls.ROW_MAJOR, 300, 16, 16, Bd.reshape(-1))
    Cm = pls.SpMat.null(300, 16)
    pls.spmm_optimize(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, pls.SCALAR_ONE, A, B, pls.SCALAR_ZERO, Cm)
    for _ in range(3):
        assert pls.spmm_exec(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, 1.0, A, B, 0.0, Cm) == 0
    ref = spmm_ref(rp, c, v, Bd, 1.0, 0.0, None)
    assert scaled_err(Cm.export_dense(), ref, rp, c, v, Bd, 1.0, 0.0, None) <= 1e-12


def test_bsr_spmm_vs_oracle():
    rng = np.random.default_rng(9)
    for bs in (2, 4, 8, 3):
        for layout in (pls.ROW_MAJOR, pls.COL_MAJOR):
            m = n = bs * 40
            rp, c, v = W.random_csr(m, n, 12, rng)
            brp, bc, bv = oracle.csr2bsr(rp, c, v, m, n, bs, layout)
            for k in (4, 8, 64):
                Bd = rng.uniform(-1, 1, (n, k))
                A = pls.SpMat.bsr(layout, m, n, bs, brp, bc, bv)
                B = pls.SpMat.dense(pls.ROW_MAJOR, n, k, k, Bd.reshape(-1))
                Cm = pls.SpMat.null(m, k)
                assert pls.spmm_exec(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, 1.0, A, B, 0.0, Cm) == 0
                ref = spmm_ref(rp, c, v, Bd, 1.0, 0.0, None)
                assert scaled_err(Cm.export_dense(), ref, rp, c, v, Bd, 1.0, 0.0, None) <= 1e-12, (bs, layout, k)
                # BSR SpMV
                x = rng.uniform(-1, 1, n)
                y_ref = oracle.csr_spmv(rp, c, v, x)
                assert rel_err_rows(A.spmv(x), y_ref, oracle.csr_absdot(rp, c, v, x)).max() <= 1e-12


@pytest.mark.parametrize("dtype,storage", [(np.float64, pls.STORAGE_NATIVE), (np.float64, pls.STORAGE_FP32),
                                           (np.float32, pls.STORAGE_NATIVE), (np.float32, pls.STORAGE_BF16)])
def test_bsr_vector_kernel_equals_scalar_kernel_bitwise(dtype, storage):
    """The BSR FMA kernel with 16-byte vectors of B and C (ldb, ldc multiples
    of the vector) adds each element of C's products in the same order, with
    the same epilogue, as the scalar kernel that runs when the strides are
    not: the same bits, for block sizes 2 / 4 / 8, both block layouts, k
    from one vector to several passes, beta = 0 and beta != 0, empty block
    rows. Both also match the FP64 oracle."""
    import torch

    rng = np.random.default_rng(70)
    vec = 16 // np.dtype(dtype).itemsize
    tol = {pls.STORAGE_NATIVE: 1e-12 if dtype == np.float64 else 1e-5, pls.STORAGE_FP32: 1e-5,
           pls.STORAGE_BF16: 1e-2}[storage]
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    for bs in (2, 4, 8):
        for layout in (pls.ROW_MAJOR, pls.COL_MAJOR):
            mb, nb = 150, 130
            rp = np.zeros(mb + 1, np.int32)
            cols = []
            for i in range(mb):
                cnt = 0 if i % 11 == 0 else int(rng.integers(1, 7))
                cols.append(np.sort(rng.choice(nb, cnt, replace=False)))
                rp[i + 1] = rp[i] + cnt
            col = np.concatenate(cols).astype(np.int32)
            vals = rng.uniform(-1, 1, len(col) * bs * bs).astype(dtype)
            m, n = mb * bs, nb * bs
            crp, cc, cv = oracle.bsr2csr(rp, col, vals.astype(np.float64), bs, layout)
            A = pls.SpMat.bsr(layout, m, n, bs, rp, col, vals)
            A.set_storage(storage)
            A.set_spmm_path(0)  # the FMA kernel (not the tensor-core one) at bs 8 with BF16 values
            for k in (vec, 8 * vec, 48 * vec):
                Bd = rng.uniform(-1, 1, (n, k)).astype(dtype)
                C0 = rng.uniform(-1, 1, (m, k)).astype(dtype)
                B64 = Bd.astype(np.float64)
                for alpha, beta in ((1.0, 0.0), (0.75, -1.5)):
                    outs = []
                    for pad in (0, 1):  # ld = k: vector kernel; ld = k + 1: scalar kernel
                        ld = k + pad
                        Bt = torch.zeros((n, ld), dtype=tdt, device="cuda")
                        Bt[:, :k] = torch.tensor(Bd, device="cuda")
                        Ct = torch.zeros((m, ld), dtype=tdt, device="cuda")
                        Ct[:, :k] = torch.tensor(C0, device="cuda")
                        A.spmm_dev(Bt.data_ptr(), ld, k, Ct.data_ptr(), ld, alpha, beta)
                        torch.cuda.synchronize()
                        assert A.spmm_info()["path"] == 6
                        outs.append(Ct[:, :k].cpu().numpy())
                    np.testing.assert_array_equal(outs[0], outs[1], err_msg=str((bs, layout, k, beta)))
                    ref = spmm_ref(crp, cc, cv, B64, alpha, beta, C0.astype(np.float64) if beta else None)
                    err = scaled_err(outs[0].astype(np.float64), ref, crp, cc, cv, B64, alpha, beta,
                                     C0.astype(np.float64))
                    assert err <= tol, (bs, layout, k, beta, err)


@pytest.mark.parametrize("storage,tol", [(pls.STORAGE_NATIVE, 1e-12), (pls.STORAGE_FP32, 1e-5),
                                         (pls.STORAGE_BF16, 1e-2)])
def test_stencil_spmm_storage_modes(storage, tol):
    m, n, rp, c, v = W.stencil_27pt(24, seed=2)
    rng = np.random.default_rng(2)
    for k in (8, 32):
        Bd = rng.uniform(-1, 1, (n, k))
        ref = spmm_ref(rp, c, v, Bd, 1.0, 0.0, None)
        dt = np.float64 if storage == pls.STORAGE_NATIVE else np.float32
        A = pls.SpMat.csr(m, n, rp, c, v.astype(dt))
        A.set_storage(storage)
        B = pls.SpMat.dense(pls.ROW_MAJOR, n, k, k, Bd.astype(dt).reshape(-1))
        Cm = pls.SpMat.null(m, k, dtype=dt)
        assert pls.spmm_exec(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, 1.0, A, B, 0.0, Cm) == 0
        got = Cm.export_dense().astype(np.float64)
        assert scaled_err(got, ref, rp, c, v, Bd, 1.0, 0.0, None) <= tol


def test_device_pointer_spmm():
    import torch

    rng = np.random.default_rng(3)
    rp, c, v = W.random_csr(1000, 800, 30, rng)
    Bd = rng.uniform(-1, 1, (800, 32))
    A = pls.SpMat.csr(1000, 800, rp, c, v)
    Bt = torch.tensor(Bd, device="cuda")
    Ct = torch.empty((1000, 32), dtype=torch.float64, device="cuda")
    A.spmm_dev(Bt.data_ptr(), 32, 32, Ct.data_ptr(), 32, 1.0, 0.0, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    ref = spmm_ref(rp, c, v, Bd, 1.0, 0.0, None)
    assert scaled_err(Ct.cpu().numpy(), ref, rp, c, v, Bd, 1.0, 0.0, None) <= 1e-12


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_staged_spmm_vs_oracle(dt):
    """The staged (shared-memory tile) SpMM on a 27-point stencil and a
    banded matrix: one column tile (k = 8, 32), several (k = 136 FP64 /
    200 FP32: 512-byte tiles plus a partial one), beta != 0, and a strided
    B (ldb > k: per-row copies). The tiled kernel must be the one that ran."""
    import torch

    rng = np.random.default_rng(7)
    m, n, rp, c, v = W.stencil_27pt(20, seed=2)
    band = W.banded_csr(5000, 9, rng)
    tol = 1e-12 if dt == np.float64 else 1e-5
    tdt = torch.float64 if dt == np.float64 else torch.float32
    cases = [(m, n, rp, c, v), band]
    ks = (8, 24, 32, 136) if dt == np.float64 else (8, 20, 32, 200)
    for (mm, nn, rpp, cc, vv) in cases:
        vv = vv.astype(dt)
        A = pls.SpMat.csr(mm, nn, rpp, cc, vv)
        A.set_spmm_path(1)  # the staged kernel whenever it applies
        for k in ks:
            for ldb in (k, k + 8):
                Bd = rng.uniform(-1, 1, (nn, ldb)).astype(dt)
                C0 = rng.uniform(-1, 1, (mm, k)).astype(dt)
                Bt = torch.tensor(Bd, device="cuda")
                Ct = torch.tensor(C0, device="cuda")
                s = torch.cuda.Stream()
                A.spmm_dev(Bt.data_ptr(), ldb, k, Ct.data_ptr(), k, 1.25, -0.5, s.cuda_stream)
                s.synchronize()
                info = A.spmm_info()
                assert info["tile_rows"] > 0 and info["path"] == 1, (mm, k, ldb, info)
                got = Ct.cpu().numpy().astype(np.float64)
                B64 = np.ascontiguousarray(Bd[:, :k].astype(np.float64))
                v64 = vv.astype(np.float64)
                ref = spmm_ref(rpp, cc, v64, B64, 1.25, -0.5, C0.astype(np.float64))
                err = scaled_err(got, ref, rpp, cc, v64, B64, 1.25, -0.5, C0.astype(np.float64))
                assert err <= tol, (mm, k, ldb, err)


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_shared_entries_spmm_vs_oracle(dt):
    """The row-group kernel with shared entry loads (a row's lanes load its
    entries together and pass them round): ragged rows with empty ones in
    one warp (the warp runs to its longest row), a stencil, a band; aligned
    and unaligned k, beta != 0. Each result matches the oracle within the
    tolerance, and equals the plain row-group kernel's bit for bit where
    that kernel also keeps each row's nonzeros in one lane (same summation
    order)."""
    import torch

    rng = np.random.default_rng(11)
    tol = 1e-12 if dt == np.float64 else 1e-5
    tdt = torch.float64 if dt == np.float64 else torch.float32
    rpr, cr, vr = W.random_csr(3000, 2000, 60, rng, empty_frac=0.3)
    cases = [(3000, 2000, rpr, cr, vr), W.stencil_27pt(12, seed=2), W.banded_csr(4000, 7, rng)]
    for (m, n, rp, c, v) in cases:
        v = v.astype(dt)
        A = pls.SpMat.csr(m, n, rp, c, v)
        for k in (8, 13, 32, 72, 130):
            Bd = rng.uniform(-1, 1, (n, k)).astype(dt)
            C0 = rng.uniform(-1, 1, (m, k)).astype(dt)
            Bt = torch.tensor(Bd, device="cuda")
            out = {}
            for path in (0, 2):
                A.set_spmm_path(path)
                Ct = torch.tensor(C0, device="cuda")
                torch.cuda.synchronize()
                A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.25, -0.5)
                torch.cuda.synchronize()
                out[path] = (Ct.cpu().numpy(), A.spmm_info()["path"])
            # Shared entries need at least 4 column lanes per row; the vector
            # width is halved until there are (FP32 k = 8: 4 lanes of 2).
            assert out[2][1] == 2, (m, k, out[2][1])
            vec = 16 // np.dtype(dt).itemsize
            cols = -(-k // vec) if k % vec == 0 else k
            if cols > 2:  # the plain kernel also gives each row one lane group (TN = 1)
                np.testing.assert_array_equal(out[0][0], out[2][0])
            v64, B64, C064 = v.astype(np.float64), Bd.astype(np.float64), C0.astype(np.float64)
            ref = spmm_ref(rp, c, v64, B64, 1.25, -0.5, C064)
            assert scaled_err(out[2][0].astype(np.float64), ref, rp, c, v64, B64, 1.25, -0.5,
                              C064) <= tol, (m, k)
        A.destroy()


def test_random_matrix_keeps_row_group_kernel():
    """B rows of a random matrix are not reused within row blocks: the
    staged path declines and a row-group kernel (plain or with shared
    entries, whichever measured faster) gives the result."""
    rng = np.random.default_rng(8)
    rp, c, v = W.random_csr(3000, 3000, 20, rng)
    Bd = rng.uniform(-1, 1, (3000, 32))
    A = pls.SpMat.csr(3000, 3000, rp, c, v)
    B = pls.SpMat.dense(pls.ROW_MAJOR, 3000, 32, 32, Bd.reshape(-1))
    Cm = pls.SpMat.null(3000, 32)
    assert pls.spmm_exec(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, 1.0, A, B, 0.0, Cm) == 0
    info = A.spmm_info()
    assert info["tile_rows"] == 0 and info["path"] in (0, 2), info
    ref = spmm_ref(rp, c, v, Bd, 1.0, 0.0, None)
    assert scaled_err(Cm.export_dense(), ref, rp, c, v, Bd, 1.0, 0.0, None) <= 1e-12


def test_spmm_measured_choice_matches_oracle():
    """Default path: the first SpMM times the applicable kernels on scratch
    output, keeps the fastest, and the result matches the oracle (beta != 0:
    the timing runs must not touch C). On a stencil the diagonal forms are
    timed and the staged kernel is not; on a band of 41 diagonals (beyond
    the diagonal form's 32) the staged kernel is timed."""
    import torch

    rng = np.random.default_rng(11)
    cases = [(W.stencil_27pt(24, seed=2), False), (W.banded_csr(20000, 20, rng), True)]
    for (m, n, rp, c, v), staged_timed in cases:
        A = pls.SpMat.csr(m, n, rp, c, v)
        for k in (8, 32):
            Bd = rng.uniform(-1, 1, (n, k))
            C0 = rng.uniform(-1, 1, (m, k))
            Bt, Ct = torch.tensor(Bd, device="cuda"), torch.tensor(C0, device="cuda")
            s = torch.cuda.Stream()
            A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 0.75, 1.5, s.cuda_stream)
            s.synchronize()
            info = A.spmm_info()
            assert info["ms_rows"] > 0, info
            if staged_timed:
                assert info["path"] in (0, 1, 2) and info["ms_staged"] > 0, info
            else:
                assert info["path"] in (0, 2, 3, 4) and info["ms_staged"] == 0, info
            ref = spmm_ref(rp, c, v, Bd, 0.75, 1.5, C0)
            assert scaled_err(Ct.cpu().numpy(), ref, rp, c, v, Bd, 0.75, 1.5, C0) <= 1e-12


@pytest.mark.parametrize("ta", [pls.OPERATION_NOTRANS, pls.OPERATION_TRANS])
@pytest.mark.parametrize("tb", [pls.OPERATION_NOTRANS, pls.OPERATION_TRANS])
def test_dense_times_sparse_vs_numpy(ta, tb):
    """Dense x sparse through the (AB)^T = B^T A^T identity of the reference
    (src/matmul.cpp:654-740): C = alpha op(A) op(B) + beta C with A dense
    (row- or column-major), B sparse CSR, C null or dense of either layout;
    m = 3 takes the narrow (one SpMV per column) path inside."""
    rng = np.random.default_rng(31 + 2 * ta + tb)
    for m, kk, n in [(40, 60, 50), (3, 30, 20)]:
        bm, bn = (kk, n) if tb == pls.OPERATION_NOTRANS else (n, kk)
        brp, bc, bv = W.random_csr(bm, bn, 8, rng)
        Bsp = np.zeros((bm, bn))
        for i in range(bm):
            Bsp[i, bc[brp[i]:brp[i + 1]]] = bv[brp[i]:brp[i + 1]]
        opB = Bsp if tb == pls.OPERATION_NOTRANS else Bsp.T
        am, an = (m, kk) if ta == pls.OPERATION_NOTRANS else (kk, m)
        Ad = rng.uniform(-1, 1, (am, an))
        opA = Ad if ta == pls.OPERATION_NOTRANS else Ad.T
        for a_layout in (pls.ROW_MAJOR, pls.COL_MAJOR):
            for c_kind in ("null", pls.ROW_MAJOR, pls.COL_MAJOR):
                C0 = rng.uniform(-1, 1, (m, n))
                beta = 0.0 if c_kind == "null" else -0.75
                A = pls.SpMat.dense(a_layout, am, an, an if a_layout == pls.ROW_MAJOR else am,
                                    (Ad if a_layout == pls.ROW_MAJOR else Ad.T).reshape(-1))
                B = pls.SpMat.csr(bm, bn, brp, bc, bv)
                if c_kind == "null":
                    Cm = pls.SpMat.null(m, n)
                else:
                    Cm = pls.SpMat.dense(c_kind, m, n, n if c_kind == pls.ROW_MAJOR else m,
                                         (C0 if c_kind == pls.ROW_MAJOR else C0.T).reshape(-1))
                st = pls.spmm_exec(ta, tb, 1.25, A, B, beta, Cm)
                assert st == 0, (m, a_layout, c_kind)
                got = Cm.export_dense()
                ref = 1.25 * opA @ opB + beta * C0
                scale = 1.25 * np.abs(opA) @ np.abs(opB) + abs(beta) * np.abs(C0)
                assert (np.abs(got - ref) / np.maximum(scale, 1e-300)).max() <= 1e-12, (m, a_layout, c_kind)


def test_dense_times_sparse_fp32():
    rng = np.random.default_rng(41)
    m, kk, n = 64, 80, 48
    brp, bc, bv = W.random_csr(kk, n, 6, rng)
    bv = bv.astype(np.float32)
    Bsp = np.zeros((kk, n))
    for i in range(kk):
        Bsp[i, bc[brp[i]:brp[i + 1]]] = bv[brp[i]:brp[i + 1]]
    Ad = rng.uniform(-1, 1, (m, kk)).astype(np.float32)
    A = pls.SpMat.dense(pls.ROW_MAJOR, m, kk, kk, Ad.reshape(-1))
    B = pls.SpMat.csr(kk, n, brp, bc, bv)
    Cm = pls.SpMat.null(m, n, dtype=np.float32)
    assert pls.spmm_exec(pls.OPERATION_NOTRANS, pls.OPERATION_NOTRANS, 1.0, A, B, 0.0, Cm) == 0
    got = Cm.export_dense().astype(np.float64)
    ref = Ad.astype(np.float64) @ Bsp
    scale = np.abs(Ad.astype(np.float64)) @ np.abs(Bsp)
    assert (np.abs(got - ref) / np.maximum(scale, 1e-300)).max() <= 1e-5


def test_staged_wait_timeout_is_reported_and_recoverable():
    """Failure path without a fault: the test hook makes the staged kernel's
    barrier expect 16 bytes more than it copies, so its bounded wait runs out
    (20,000 polls, several milliseconds; every copy has landed by then). The
    kernel flags the failure and leaves C untouched; the handle's next SpMM
    reports EXECUTION_FAILURE; after the hook is cleared the same handle and
    context compute correctly again."""
    import torch

    m, n, rp, c, v = W.stencil_27pt(16, seed=2)
    k = 8
    rng = np.random.default_rng(12)
    Bd = rng.uniform(-1, 1, (n, k))
    A = pls.SpMat.csr(m, n, rp, c, v)
    A.set_spmm_path(1)
    Bt = torch.tensor(Bd, device="cuda")
    Ct = torch.full((m, k), 7.0, dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    L = pls.lib()
    assert L.perflibs_b200_testing_stage_fault(16, 20000) == 0
    try:
        A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0, s.cuda_stream)
        s.synchronize()
        assert A.spmm_info()["path"] == 1
        assert torch.all(Ct == 7.0)  # C untouched by the failed launch
        with pytest.raises(pls.PerflibsError) as e:
            A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0, s.cuda_stream)
        assert e.value.status == pls.STATUS_EXECUTION_FAILURE
    finally:
        assert L.perflibs_b200_testing_stage_fault(0, 0) == 0
    s.synchronize()
    A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0, s.cuda_stream)
    s.synchronize()
    ref = spmm_ref(rp, c, v, Bd, 1.0, 0.0, None)
    assert scaled_err(Ct.cpu().numpy(), ref, rp, c, v, Bd, 1.0, 0.0, None) <= 1e-12


def test_dia_tma_wait_timeout_is_reported_and_recoverable():
    """The same failure path for the diagonal form with TMA-staged B: its
    window barriers expect 16 bytes more than the tensor copies bring, so
    every CTA's bounded wait runs out with all copies landed; C is left
    untouched, the next SpMM reports EXECUTION_FAILURE, and once the hook is
    cleared the handle computes correctly."""
    import torch

    m, n, rp, c, v = W.stencil_27pt(16, seed=2)
    k = 8
    rng = np.random.default_rng(13)
    Bd = rng.uniform(-1, 1, (n, k))
    A = pls.SpMat.csr(m, n, rp, c, v)
    A.set_spmm_path(4)
    Bt = torch.tensor(Bd, device="cuda")
    Ct = torch.full((m, k), 7.0, dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    L = pls.lib()
    assert L.perflibs_b200_testing_stage_fault(16, 20000) == 0
    try:
        A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0, s.cuda_stream)
        s.synchronize()
        assert A.spmm_info()["path"] == 4
        assert torch.all(Ct == 7.0)
        with pytest.raises(pls.PerflibsError) as e:
            A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0, s.cuda_stream)
        assert e.value.status == pls.STATUS_EXECUTION_FAILURE
    finally:
        assert L.perflibs_b200_testing_stage_fault(0, 0) == 0
    s.synchronize()
    A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0, s.cuda_stream)
    s.synchronize()
    assert A.spmm_info()["path"] == 4
    ref = spmm_ref(rp, c, v, Bd, 1.0, 0.0, None)
    assert scaled_err(Ct.cpu().numpy(), ref, rp, c, v, Bd, 1.0, 0.0, None) <= 1e-12


@pytest.mark.parametrize("storage", [pls.STORAGE_NATIVE, pls.STORAGE_FP32, pls.STORAGE_BF16])
def test_dia_tma_equals_diagonal_form_bitwise(storage):
    """The diagonal form with TMA-staged B adds each row's entries in the
    same order with the same arithmetic as the diagonal-form kernel, so the
    two agree bit for bit: 27- and 7-point 3-D stencils (windows chained
    over planes), 5- and 9-point 2-D stencils (over lines), bands and a
    diagonal (one group); k from one 16-byte vector to several column
    slices with a partial last one (the staged kernel runs from four vectors
    on; narrower k may not fit its windows in shared memory, and then the
    diagonal form runs); B with ldb > k; beta = 0 and beta != 0; and the
    result matches the oracle within the storage mode's tolerance."""
    import torch

    from tests.conftest import rel_err_rows  # noqa: F401

    rng = np.random.default_rng(21)
    native = storage == pls.STORAGE_NATIVE
    dt = np.float64 if native else np.float32
    tdt = torch.float64 if native else torch.float32
    tol = {pls.STORAGE_NATIVE: 1e-12, pls.STORAGE_FP32: 1e-5, pls.STORAGE_BF16: 1e-2}[storage]

    def stencil(g, pts):
        if pts == 27:
            return W.stencil_27pt(g, seed=3)
        n = g ** 3 if pts == 7 else g * g
        idx = np.arange(n)
        if pts == 7:
            z, y, x = idx // (g * g), (idx // g) % g, idx % g
            nb = [(-g * g, z > 0), (-g, y > 0), (-1, x > 0), (0, idx >= 0), (1, x < g - 1), (g, y < g - 1),
                  (g * g, z < g - 1)]
        else:
            y, x = idx // g, idx % g
            nb = [(dy * g + dx, (y + dy >= 0) & (y + dy < g) & (x + dx >= 0) & (x + dx < g))
                  for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
        cols = np.stack([idx + o for o, _ in nb], 1)
        mask = np.stack([mk for _, mk in nb], 1)
        rp = np.zeros(n + 1, np.int32)
        rp[1:] = np.cumsum(mask.sum(1))
        return n, n, rp, cols[mask].astype(np.int32), rng.uniform(-1, 1, int(rp[-1]))

    cases = [stencil(22, 27), stencil(30, 7), stencil(150, 9), W.laplacian_2d(200),
             W.banded_csr(7001, 6, rng), W.banded_csr(513, 0, rng)]
    for (m, n, rp, c, v) in cases:
        A = pls.SpMat.csr(m, n, rp, c, v.astype(dt))
        A.set_storage(storage)
        for k in (4, 8, 16, 24, 40, 72, 136):
            vec = 16 // np.dtype(dt).itemsize
            if k % vec:
                continue
            for ldb in (k, k + 2 * vec):
                Bd = rng.uniform(-1, 1, (n, ldb)).astype(dt)
                C0 = rng.uniform(-1, 1, (m, k)).astype(dt)
                Bt = torch.tensor(Bd, device="cuda")
                for alpha, beta in ((1.5, 0.0), (-0.75, 0.5)):
                    outs = {}
                    for path in (3, 4):
                        A.set_spmm_path(path)
                        Ct = torch.tensor(C0, device="cuda")
                        A.spmm_dev(Bt.data_ptr(), ldb, k, Ct.data_ptr(), k, alpha, beta)
                        torch.cuda.synchronize()
                        outs[path] = (Ct.cpu().numpy(), A.spmm_info()["path"])
                    # path 4 falls back to the diagonal form when its plan does not fit
                    # shared memory (k of one or two vectors on the 3-D stencil)
                    assert outs[3][1] == 3 and outs[4][1] in (3, 4), (m, k, ldb, outs[3][1], outs[4][1])
                    if k >= 4 * vec:
                        assert outs[4][1] == 4, (m, k, ldb)
                    np.testing.assert_array_equal(outs[4][0], outs[3][0], err_msg=f"m={m} k={k} ldb={ldb}")
                    B64 = np.ascontiguousarray(Bd[:, :k].astype(np.float64))
                    ref = spmm_ref(rp, c, v, B64, alpha, beta, C0.astype(np.float64) if beta else None)
                    err = scaled_err(outs[4][0].astype(np.float64), ref, rp, c, v, B64, alpha, beta,
                                     C0.astype(np.float64))
                    assert err <= tol, (m, k, ldb, err)


def _laplacian_rect(nx, ny, rng):
    """5-point operator on an nx x ny grid (rows of nx points: the line stride
    is nx), random values, sorted columns."""
    n = nx * ny
    i = np.arange(n, dtype=np.int64)
    r, c = i // nx, i % nx
    offs = [(-nx, r > 0), (-1, c > 0), (0, np.ones(n, bool)), (1, c < nx - 1), (nx, r < ny - 1)]
    cols = np.stack([i + o for o, _ in offs], 1)
    mask = np.stack([mk for _, mk in offs], 1)
    counts = mask.sum(1)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(counts)
    col = cols[mask].astype(np.int32)
    return n, n, rp, col, rng.uniform(-1, 1, len(col))


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_diagonal_form_line_patches_equal_row_group_bitwise(dt):
    """Grids whose line stride lets the diagonal-form kernel give each CTA a
    patch of 4 grid lines (64-point lines; a 27-point stencil on 32^3 and
    64^3), with a tail of units past the last whole group of lines (37 and 41
    lines): with beta = 0 the kernel must equal the row-group kernel bit for
    bit at every column count (1, several or many lanes per unit, one or two
    passes), so every row is computed once by the right thread, and match the
    oracle."""
    import torch

    rng = np.random.default_rng(23)
    vec = 16 // np.dtype(dt).itemsize
    tol = 1e-12 if dt == np.float64 else 1e-5
    cases = [_laplacian_rect(64, 37, rng), _laplacian_rect(64, 41, rng), W.stencil_27pt(32, seed=5),
             W.stencil_27pt(64, seed=6)]
    for (m, n, rp, c, v) in cases:
        v = v.astype(dt)
        A = pls.SpMat.csr(m, n, rp, c, v)
        for k in (8, 32, 64, 128, 256):
            Bd = rng.uniform(-1, 1, (n, k)).astype(dt)
            Bt = torch.tensor(Bd, device="cuda")
            out = {}
            for path in (0, 3):
                A.set_spmm_path(path)
                Ct = torch.full((m, k), float("nan"), dtype=Bt.dtype, device="cuda")
                A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0)
                torch.cuda.synchronize()
                out[path] = (Ct.cpu().numpy(), A.spmm_info()["path"])
            assert out[3][1] == 3, (m, k)
            if k // vec > 2:  # the row-group kernel also keeps each row in one lane group
                np.testing.assert_array_equal(out[0][0], out[3][0], err_msg=str((m, k)))
            v64, B64 = v.astype(np.float64), Bd.astype(np.float64)
            Z = np.zeros((m, k))
            assert scaled_err(out[3][0].astype(np.float64), spmm_ref(rp, c, v64, B64, 1.0, 0.0, Z),
                              rp, c, v64, B64, 1.0, 0.0, Z) <= tol, (m, k)
        A.destroy()


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_diagonal_form_spmm(dt):
    """The diagonal-form SpMM (entries on a few diagonals, kept per block of
    rows with absent entries skipped). On a 27-point stencil, a 2D Laplacian
    and a narrow band it takes the diagonal path and equals the row-group
    kernel bit for bit with beta = 0 (same entries, same ascending order,
    one fma each); with beta != 0 it matches the oracle. A NaN in a row of B
    reaches exactly the rows that store an entry in that column. A random
    matrix does not qualify and keeps the row-group kernel. After the
    values are updated, the diagonal form is rebuilt from the new values."""
    import torch

    rng = np.random.default_rng(17)
    tol = 1e-12 if dt == np.float64 else 1e-5
    vec = 16 // np.dtype(dt).itemsize
    cases = [W.stencil_27pt(10, seed=2), W.laplacian_2d(37), W.banded_csr(3001, 3, rng)]
    for (m, n, rp, c, v) in cases:
        v = v.astype(dt)
        A = pls.SpMat.csr(m, n, rp, c, v)
        for k in (vec, 8, 32, 40, 136):
            if k % vec:
                continue
            Bd = rng.uniform(-1, 1, (n, k)).astype(dt)
            C0 = rng.uniform(-1, 1, (m, k)).astype(dt)
            Bt = torch.tensor(Bd, device="cuda")
            out = {}
            for path in (0, 3):
                A.set_spmm_path(path)
                Ct = torch.zeros((m, k), dtype=Bt.dtype, device="cuda")
                torch.cuda.synchronize()
                A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0)
                torch.cuda.synchronize()
                out[path] = (Ct.cpu().numpy(), A.spmm_info()["path"])
            assert out[3][1] == 3, (m, k)
            v64, B64 = v.astype(np.float64), Bd.astype(np.float64)
            if k // vec > 2:  # the row-group kernel also keeps each row in one lane group
                np.testing.assert_array_equal(out[0][0], out[3][0])
            Z = np.zeros((m, k))
            assert scaled_err(out[3][0].astype(np.float64), spmm_ref(rp, c, v64, B64, 1.0, 0.0, Z),
                              rp, c, v64, B64, 1.0, 0.0, Z) <= tol, (m, k)
            Ct = torch.tensor(C0, device="cuda")
            A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.25, -0.5)
            torch.cuda.synchronize()
            v64, B64, C064 = v.astype(np.float64), Bd.astype(np.float64), C0.astype(np.float64)
            ref = spmm_ref(rp, c, v64, B64, 1.25, -0.5, C064)
            assert scaled_err(Ct.cpu().numpy().astype(np.float64), ref, rp, c, v64, B64, 1.25, -0.5,
                              C064) <= tol, (m, k)
        # a NaN in one row of B reaches the rows with an entry in that column
        k = 2 * vec
        Bd = rng.uniform(-1, 1, (n, k)).astype(dt)
        j = n // 2
        Bd[j, :] = np.nan
        Bt = torch.tensor(Bd, device="cuda")
        Ct = torch.zeros((m, k), dtype=Bt.dtype, device="cuda")
        A.set_spmm_path(3)
        A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0)
        torch.cuda.synchronize()
        assert A.spmm_info()["path"] == 3
        rows_with_j = np.unique(np.repeat(np.arange(m), np.diff(rp))[c == j])
        nan_rows = np.where(np.isnan(Ct.cpu().numpy()).any(axis=1))[0]
        np.testing.assert_array_equal(nan_rows, rows_with_j)
        # updated values: the diagonal form is built again
        k = 8 if vec <= 8 else vec
        Bd = rng.uniform(-1, 1, (n, k)).astype(dt)
        Bt = torch.tensor(Bd, device="cuda")
        rows = np.repeat(np.arange(m), np.diff(rp))[::5].astype(np.int32)
        assert A.update(rows, c[::5].astype(np.int32), np.full(len(rows), 2.5, dt)) == 0
        v2 = v.astype(np.float64)
        v2[::5] = 2.5
        Ct = torch.zeros((m, k), dtype=Bt.dtype, device="cuda")
        A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0)
        torch.cuda.synchronize()
        assert A.spmm_info()["path"] == 3
        ref = spmm_ref(rp, c, v2, Bd.astype(np.float64), 1.0, 0.0, np.zeros((m, k)))
        assert scaled_err(Ct.cpu().numpy().astype(np.float64), ref, rp, c, v2, Bd.astype(np.float64),
                          1.0, 0.0, np.zeros((m, k))) <= tol
        A.destroy()
    # reduced value storage (FP32 / BF16 values, FP32 accumulation): the
    # diagonal form keeps the stored values and sums like the row-group kernel
    m, n, rp, c, v = W.stencil_27pt(9, seed=4)
    A = pls.SpMat.csr(m, n, rp, c, v.astype(dt))
    k = 32
    Bd = rng.uniform(-1, 1, (n, k)).astype(dt)
    Bt = torch.tensor(Bd, device="cuda")
    storages = [pls.STORAGE_BF16] + ([pls.STORAGE_FP32] if dt == np.float64 else [])
    for storage in storages:
        A.set_storage(storage)
        out = {}
        for path in (0, 3):
            A.set_spmm_path(path)
            Ct = torch.zeros((m, k), dtype=Bt.dtype, device="cuda")
            A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0)
            torch.cuda.synchronize()
            out[path] = (Ct.cpu().numpy(), A.spmm_info()["path"])
        assert out[3][1] == 3, storage
        np.testing.assert_array_equal(out[0][0], out[3][0])
    A.destroy()
    # a random matrix has no diagonal form: the forced path falls back
    rp, c, v = W.random_csr(2000, 2000, 20, rng)
    A = pls.SpMat.csr(2000, 2000, rp, c, v.astype(dt))
    A.set_spmm_path(3)
    Bt = torch.tensor(rng.uniform(-1, 1, (2000, 8)).astype(dt), device="cuda")
    Ct = torch.zeros((2000, 8), dtype=Bt.dtype, device="cuda")
    A.spmm_dev(Bt.data_ptr(), 8, 8, Ct.data_ptr(), 8, 1.0, 0.0)
    torch.cuda.synchronize()
    assert A.spmm_info()["path"] == 0
    A.destroy()


def _random_bsr8(rng, mb, nb, max_blocks, layout, empty_frac=0.1):
    """Random BSR with 8 x 8 blocks: 0 .. max_blocks distinct block columns
    per block row (some rows empty), FP32 values U[-1, 1] with about 20% of
    the entries explicit zeros."""
    rp = np.zeros(mb + 1, np.int32)
    cols = []
    for i in range(mb):
        cnt = 0 if rng.random() < empty_frac else int(rng.integers(1, max_blocks + 1))
        c = np.sort(rng.choice(nb, min(cnt, nb), replace=False))
        cols.append(c)
        rp[i + 1] = rp[i] + len(c)
    col = np.concatenate(cols).astype(np.int32)
    vals = rng.uniform(-1, 1, len(col) * 64).astype(np.float32)
    vals[rng.random(len(vals)) < 0.2] = 0.0
    return rp, col, vals


@pytest.mark.parametrize("layout", [pls.ROW_MAJOR, pls.COL_MAJOR])
def test_bsr_tensor_core_spmm_vs_oracle(layout):
    """The tensor-core BSR SpMM (tcgen05.mma kind::tf32, bs = 8, BF16 value
    storage, FP32 B and C): every k from one column chunk of 128 to several
    with a partial last one, B with ldb > k, beta = 0 and beta != 0, empty
    block rows. Forced (path 5) it must run and match the FP64 oracle of the
    FP32 values within the BF16 storage mode's 1e-2 (scaled per element),
    as the FMA kernel does; the measured choice (path -1) picks one of the
    two and is correct too."""
    import torch

    rng = np.random.default_rng(40 + layout)
    mb, nb = 300, 260
    rp, col, vals = _random_bsr8(rng, mb, nb, 12, layout)
    m, n = mb * 8, nb * 8
    crp, cc, cv = oracle.bsr2csr(rp, col, vals.astype(np.float64), 8, layout)
    A = pls.SpMat.bsr(layout, m, n, 8, rp, col, vals)
    A.set_storage(pls.STORAGE_BF16)
    for k in (8, 64, 128, 200, 256):
        for ldb in (k, k + 12):
            Bd = rng.uniform(-1, 1, (n, ldb)).astype(np.float32)
            C0 = rng.uniform(-1, 1, (m, k)).astype(np.float32)
            Bt = torch.tensor(Bd, device="cuda")
            B64 = np.ascontiguousarray(Bd[:, :k].astype(np.float64))
            for alpha, beta in ((1.0, 0.0), (-0.5, 0.75)):
                ref = spmm_ref(crp, cc, cv, B64, alpha, beta, C0.astype(np.float64) if beta else None)
                for path, expect in ((5, 5), (0, 6), (-1, None)):
                    A.set_spmm_path(path)
                    Ct = torch.tensor(C0, device="cuda")
                    A.spmm_dev(Bt.data_ptr(), ldb, k, Ct.data_ptr(), k, alpha, beta)
                    torch.cuda.synchronize()
                    ran = A.spmm_info()["path"]
                    assert ran == expect if expect else ran in (5, 6), (k, ldb, path, ran)
                    got = Ct.cpu().numpy().astype(np.float64)
                    err = scaled_err(got, ref, crp, cc, cv, B64, alpha, beta, C0.astype(np.float64))
                    assert err <= 1e-2, (k, ldb, path, err)


def test_bsr_tensor_core_wait_timeout_is_reported_and_recoverable():
    """Failure path of the tensor-core BSR kernel without a fault: with the
    test hook armed, each CTA's first wait for a finished accumulator goes to
    a barrier that nothing arrives on, so the bounded wait runs out; the
    CTAs stop, wait for their MMAs in flight and free their tensor memory; C
    is untouched, the next SpMM reports EXECUTION_FAILURE, and with the hook
    cleared the handle computes correctly."""
    import torch

    rng = np.random.default_rng(77)
    # no empty block rows: every CTA's first epilogue waits for an accumulator
    rp, col, vals = _random_bsr8(rng, 64, 64, 4, pls.ROW_MAJOR, empty_frac=0.0)
    A = pls.SpMat.bsr(pls.ROW_MAJOR, 512, 512, 8, rp, col, vals)
    A.set_storage(pls.STORAGE_BF16)
    A.set_spmm_path(5)
    k = 64
    Bd = rng.uniform(-1, 1, (512, k)).astype(np.float32)
    Bt = torch.tensor(Bd, device="cuda")
    Ct = torch.full((512, k), 7.0, dtype=torch.float32, device="cuda")
    L = pls.lib()
    assert L.perflibs_b200_testing_stage_fault(16, 20000) == 0
    try:
        A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0)
        torch.cuda.synchronize()
        assert A.spmm_info()["path"] == 5
        assert torch.all(Ct == 7.0)
        with pytest.raises(pls.PerflibsError) as e:
            A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0)
        assert e.value.status == pls.STATUS_EXECUTION_FAILURE
    finally:
        assert L.perflibs_b200_testing_stage_fault(0, 0) == 0
    torch.cuda.synchronize()
    A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0)
    torch.cuda.synchronize()
    assert A.spmm_info()["path"] == 5
    crp, cc, cv = oracle.bsr2csr(rp, col, vals.astype(np.float64), 8, pls.ROW_MAJOR)
    B64 = Bd.astype(np.float64)
    ref = spmm_ref(crp, cc, cv, B64, 1.0, 0.0, None)
    assert scaled_err(Ct.cpu().numpy().astype(np.float64), ref, crp, cc, cv, B64, 1.0, 0.0, None) <= 1e-2
