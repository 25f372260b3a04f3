"""GPU parity: SpMV through the C-ABI against the oracle and the reference's
golden vectors.

Tolerance (FP64 drop-in path): per-row |y - y_ref| / max(|y_ref|, s_i)
<= 1e-12, s_i = |alpha| sum_j |a_ij x_j| + |beta| |y0_i| — the only
difference allowed is the order of the row's summation.
"""
import numpy as np
import pytest

import oracle
import perf_libs_sparse_b200 as pls
from perf_libs_sparse_b200 import workloads as W
from tests.conftest import case_names, rel_err_rows

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def scale_of(rp, c, v, x, alpha, beta, y0):
    s = abs(alpha) * oracle.csr_absdot(rp, c, v, x)
    if y0 is not None and beta != 0:
        s = s + abs(beta) * np.abs(y0)
    return s


def configs():
    out = [(pls.KIND_CSR, 0, 0, t) for t in (1, 2, 4, 8, 16, 32)]
    out.append((pls.KIND_CSR_SPLIT, 0, 0, 16))
    for C in (8, 16, 32):
        for sigma in (0, C, 4 * C, 256 if 256 % C == 0 else 0):
            out.append((pls.KIND_SELL, C, sigma, 0))
    return out


def gpu_spmv(rp, c, v, m, n, x, y0, alpha, beta, cfg=None, storage=None):
    A = pls.SpMat.csr(m, n, rp, c, v)
    if storage is not None:
        assert A.set_storage(storage) == 0
    if cfg is not None:
        assert A.force_config(*cfg) == 0
    assert A.optimize() == 0
    y = A.spmv(x, None if y0 is None else y0.copy(), alpha=alpha, beta=beta)
    A.destroy()
    return y


# ---------------------------------------------------------------- KATs


def test_kat_spmv_basic(kats):
    k = kats["spmv_basic_d"]
    A = pls.SpMat.csr(k["m"], k["n"], np.array(k["row_ptr"]), np.array(k["col"]),
                      np.array(k["vals"], np.float64))
    assert A.hint(pls.HINT_STRUCTURE, pls.STRUCTURE_UNSTRUCTURED) == 0
    assert A.hint(pls.HINT_SPMV_OPERATION, pls.OPERATION_NOTRANS) == 0
    assert A.hint(pls.HINT_SPMV_INVOCATIONS, pls.INVOCATIONS_MANY) == 0
    assert A.optimize() == 0
    y = A.spmv(np.array(k["x"], np.float64), alpha=k["alpha"], beta=k["beta"])
    np.testing.assert_allclose(y, k["y"], atol=k["tol"])


def test_kat_bsr(kats):
    k = kats["bsr_row_major"]
    A = pls.SpMat.bsr(k["layout"], k["m"], k["n"], k["bs"], np.array(k["row_ptr"]),
                      np.array(k["col"]), np.array(k["vals"], np.float64))
    x = np.array(k["x"], np.float64)
    np.testing.assert_allclose(A.spmv(x), k["y_notrans"], atol=k["tol"])
    np.testing.assert_allclose(A.spmv(x, trans=pls.OPERATION_TRANS), k["y_trans"], atol=k["tol"])
    k = kats["bsr_col_major"]
    A = pls.SpMat.bsr(k["layout"], k["m"], k["n"], k["bs"], np.array(k["row_ptr"]),
                      np.array(k["col"]), np.array(k["vals"], np.float64))
    assert A.norm(pls.NORM_INF) == k["inf_norm"]
    d = A.export_dense(pls.ROW_MAJOR)
    assert d.shape == (4, 4)
    y = A.spmv(np.array(k["x"], np.float64), alpha=k["alpha_trans"], trans=pls.OPERATION_TRANS)
    np.testing.assert_allclose(y, k["y_trans_scaled"], atol=k["tol"])


def test_kat_strategy_paths(kats):
    """Large regular matrix, optimize (tuned), export, exec, update, alpha/beta."""
    k = kats["strategy_paths_d"]
    m, w, n = k["m"], k["width"], k["n"]
    rp = (np.arange(m + 1) * w).astype(np.int32)
    col = (16 * np.arange(m)[:, None] + np.arange(w)[None, :]).reshape(-1).astype(np.int32)
    vals = np.ones(m * w)
    A = pls.SpMat.csr(m, n, rp, col, vals)
    A.hint(pls.HINT_SPMV_OPERATION, pls.OPERATION_NOTRANS)
    A.hint(pls.HINT_SPMV_INVOCATIONS, pls.INVOCATIONS_MANY)
    assert A.optimize() == 0
    mo, no, rpo, co, vo = A.export_csr(0)
    assert (mo, no) == (m, n)
    assert rpo[m] == m * w and co[0] == k["col_first"] and co[-1] == n - k["col_last_from_end"]
    x = np.ones(n)
    np.testing.assert_allclose(A.spmv(x), np.full(m, k["y_plain"]), atol=k["tol"])
    r = k["updated_row"]
    assert A.update([r], [16 * r], [2.0]) == 0
    y = A.spmv(x)
    exp = np.full(m, k["y_plain"])
    exp[r] = k["y_updated_row"]
    np.testing.assert_allclose(y, exp, atol=k["tol"])
    y = A.spmv(x, np.full(m, k["y0"]), alpha=k["alpha"], beta=k["beta"])
    np.testing.assert_allclose(y, k["alpha"] * exp + k["y0"], atol=k["tol"])


def test_kat_csr_irregular_float(kats):
    k = kats["csr_spmv_omp_paths_float"]
    m, n = k["m"], k["n"]
    cyc = k["row_lengths_cycle"]
    lens = np.array([cyc[i % 8] for i in range(m)])
    rp = np.zeros(m + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    col = np.concatenate([(29 * i + 17) % (n - lens[i]) + np.arange(lens[i]) for i in range(m)]).astype(np.int32)
    vals = (0.125 * ((np.arange(rp[-1]) % 13) + 1)).astype(np.float32)
    x = (((np.arange(n) % 11) - 5) * 0.5).astype(np.float32)
    y0 = ((np.arange(m) % 9) - 4).astype(np.float32)
    sums = np.array([np.dot(vals[rp[i]:rp[i + 1]].astype(np.float64), x[col[rp[i]:rp[i + 1]]].astype(np.float64))
                     for i in range(m)])
    exp = k["beta"] * y0 + k["alpha"] * sums.astype(np.float32)
    A = pls.SpMat.csr(m, n, rp, col, vals)
    A.hint(pls.HINT_SPMV_INVOCATIONS, pls.INVOCATIONS_MANY)
    assert A.optimize() == 0
    y = A.spmv(x, y0.copy(), alpha=k["alpha"], beta=k["beta"])
    np.testing.assert_allclose(y, exp, atol=k["tol"])


# ------------------------------------------------- fixtures of the reference


def test_reference_outputs_all_kernels(ref_outputs):
    f = ref_outputs
    for name in case_names(f):
        rp, c, v = f[f"{name}/row_ptr"], f[f"{name}/col"], f[f"{name}/vals"]
        m, n = (int(t) for t in f[f"{name}/shape"])
        x, y0, yref = f[f"{name}/x"], f[f"{name}/y0"], f[f"{name}/y_csr"]
        base = int(rp[0])
        rp0, c0 = rp - base, c - base
        sc = scale_of(rp0, c0, v, x, 1.5, -0.5, y0)
        for cfg in configs():
            y = gpu_spmv(rp, c, v, m, n, x, y0, 1.5, -0.5, cfg)
            err = rel_err_rows(y, yref, sc).max() if m else 0.0
            assert err <= FP64_TOL, (name, cfg, err)


def test_sell_layout_bit_exact_vs_reference(ref_outputs):
    f = ref_outputs
    for name in case_names(f):
        rp, c, v = f[f"{name}/row_ptr"], f[f"{name}/col"], f[f"{name}/vals"]
        m, n = (int(t) for t in f[f"{name}/shape"])
        A = pls.SpMat.csr(m, n, rp, c, v)
        for key in [k[: -len("/info")] for k in f.files if k.startswith(name + "/scs_") and k.endswith("/info")]:
            info = [int(t) for t in f[key + "/info"]]
            assert A.build_sell(info[1], info[2]) == 0
            s = A.export_sell()
            got = [s["nC"], s["C"], s["sigma"], s["col_bytes"], s["n_full_chunks"], s["ntidyup"], s["size"]]
            assert got == info, key
            for fld in ("cs", "cl", "col_min", "permd2in", "vals"):
                np.testing.assert_array_equal(s[fld], f[f"{key}/{fld}"], err_msg=f"{key}/{fld}")
            np.testing.assert_array_equal(s["offsets"], f[f"{key}/offsets"].astype(np.int64), err_msg=key)


# ------------------------------------------------------- random parity


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_vs_oracle(seed):
    rng = np.random.default_rng(100 + seed)
    for m, n, ml in [(1, 1, 1), (31, 17, 9), (300, 500, 70), (2000, 3000, 40), (5000, 5000, 300)]:
        base = int(rng.integers(0, 2))
        rp, c, v = W.random_csr(m, n, ml, rng, base=base, empty_frac=0.2)
        x = rng.uniform(-1, 1, n)
        y0 = rng.uniform(-1, 1, m)
        for alpha, beta in [(1.0, 0.0), (0.7, 1.0), (-2.0, 0.25)]:
            yref = oracle.csr_spmv(rp, c, v, x, y=y0, alpha=alpha, beta=beta)
            sc = scale_of(rp - base, c - base, v, x, alpha, beta, y0)
            for cfg in configs():
                y = gpu_spmv(rp, c, v, m, n, x, y0, alpha, beta, cfg)
                assert rel_err_rows(y, yref, sc).max() <= FP64_TOL, (m, n, cfg, alpha, beta)


def test_zipf_tail_work_list():
    """Power-law rows wide enough to trigger the sliced SELL work list."""
    m, n, rp, c, v = W.zipf_rows(200_000, seed=11)
    x = W.uniform_vector(n, 12)
    yref = oracle.csr_spmv(rp, c, v, x)
    sc = scale_of(rp, c, v, x, 1.0, 0.0, None)
    for cfg in [(pls.KIND_SELL, 32, 4096, 0), (pls.KIND_SELL, 16, 0, 0), (pls.KIND_CSR_SPLIT, 0, 0, 256),
                (pls.KIND_CSR, 0, 0, 16)]:
        y = gpu_spmv(rp, c, v, m, n, x, None, 1.0, 0.0, cfg)
        assert rel_err_rows(y, yref, sc).max() <= FP64_TOL, cfg


def test_autotune_picks_a_valid_config_and_matches():
    m, n, rp, c, v = W.zipf_rows(100_000, seed=5)
    x = W.uniform_vector(n, 6)
    A = pls.SpMat.csr(m, n, rp, c, v)
    assert A.optimize() == 0
    cfg, ms = A.tune_table()
    assert len(ms) >= 10 and np.all(ms > 0)
    y = A.spmv(x)
    yref = oracle.csr_spmv(rp, c, v, x)
    assert rel_err_rows(y, yref, scale_of(rp, c, v, x, 1, 0, None)).max() <= FP64_TOL


def test_autotune_cache_resumes_tuning(tmp_path):
    """An exhaustive tune is recorded under the matrix's structure; the same
    structure (any values) takes it from the cache without timing, across a
    save / clear / load of the cache file; another storage mode is another
    key."""
    pls.tune_cache_clear()
    m, n, rp, c, v = W.zipf_rows(60_000, seed=31)
    x = W.uniform_vector(n, 32)
    A = pls.SpMat.csr(m, n, rp, c, v)
    assert A.optimize() == 0
    assert A.tune_source() == pls.TUNE_SOURCE_TIMED
    cfg0 = A.config()
    tab_a, ms_a = A.tune_table()
    B = pls.SpMat.csr(m, n, rp, c, 2.0 * v)
    assert B.optimize() == 0
    assert B.tune_source() == pls.TUNE_SOURCE_CACHE
    assert B.config() == cfg0
    tab_b, ms_b = B.tune_table()
    np.testing.assert_array_equal(tab_a, tab_b)
    np.testing.assert_array_equal(ms_a, ms_b)
    yref = oracle.csr_spmv(rp, c, 2.0 * v, x)
    assert rel_err_rows(B.spmv(x), yref, scale_of(rp, c, 2.0 * v, x, 1, 0, None)).max() <= FP64_TOL
    F = pls.SpMat.csr(m, n, rp, c, v)
    assert F.set_storage(pls.STORAGE_FP32) == 0
    assert F.optimize() == 0
    assert F.tune_source() == pls.TUNE_SOURCE_TIMED
    path = tmp_path / "tune.cache"
    pls.tune_cache_save(path)
    assert pls.tune_cache_size() == 2
    pls.tune_cache_clear()
    D = pls.SpMat.csr(m, n, rp, c, v)
    assert D.optimize() == 0
    assert D.tune_source() == pls.TUNE_SOURCE_TIMED
    pls.tune_cache_clear()
    pls.tune_cache_load(path)
    E = pls.SpMat.csr(m, n, rp, c, v)
    assert E.optimize() == 0
    assert E.tune_source() == pls.TUNE_SOURCE_CACHE
    assert E.config() == cfg0
    tab_e, ms_e = E.tune_table()
    np.testing.assert_array_equal(tab_a, tab_e)
    np.testing.assert_allclose(ms_a, ms_e, rtol=1e-6)
    G = pls.SpMat.csr(m, n, rp, c, v)
    assert G.force_config(pls.KIND_CSR, 0, 0, 4) == 0
    assert G.optimize() == 0
    assert G.tune_source() == pls.TUNE_SOURCE_FORCED
    for h in (A, B, D, E, F, G):
        h.destroy()
    pls.tune_cache_clear()


# ------------------------------------------------------- edge cases


def test_edge_shapes_and_scalars():
    # empty matrix (m = 0), n = 0, nnz = 0
    A = pls.SpMat.csr(0, 5, np.array([0]), np.zeros(0), np.zeros(0))
    assert A.spmv(np.ones(5)).shape == (0,)
    A = pls.SpMat.csr(3, 0, np.array([0, 0, 0, 0]), np.zeros(0), np.zeros(0))
    y = A.spmv(np.zeros(0), np.array([1.0, 2.0, 3.0]), beta=2.0)
    np.testing.assert_array_equal(y, [2.0, 4.0, 6.0])
    A = pls.SpMat.csr(3, 3, np.array([0, 0, 0, 0]), np.zeros(0), np.zeros(0))
    assert A.optimize() == 0
    np.testing.assert_array_equal(A.spmv(np.ones(3), np.full(3, np.nan), beta=0.0), np.zeros(3))
    # alpha == 0: y = beta*y
    rp, c, v = np.array([0, 1, 2]), np.array([0, 1]), np.array([5.0, 7.0])
    A = pls.SpMat.csr(2, 2, rp, c, v)
    np.testing.assert_array_equal(A.spmv(np.ones(2), np.array([1.0, 2.0]), alpha=0.0, beta=3.0), [3.0, 6.0])
    # beta == 0 overwrites NaN in y
    np.testing.assert_array_equal(A.spmv(np.ones(2), np.full(2, np.nan)), [5.0, 7.0])


def test_error_codes():
    rp, c, v = np.array([0, 1]), np.array([0]), np.array([1.0])
    A = pls.SpMat.csr(-1, 1, rp, c, v, check=False)
    assert A.status == pls.STATUS_INPUT_PARAMETER_ERROR
    A = pls.SpMat.csr(1, -1, rp, c, v, check=False)
    assert A.status == pls.STATUS_INPUT_PARAMETER_ERROR
    A = pls.SpMat.csr(1, 1, np.array([2, 3]), c, v, check=False)
    assert A.status == pls.STATUS_INPUT_PARAMETER_ERROR
    A = pls.SpMat.csr(1, 1, rp, c, v)
    st, _ = A.spmv(np.ones(1), trans=999, check=False)
    assert st == pls.STATUS_INPUT_PARAMETER_ERROR
    assert A.hint(pls.HINT_SPMV_OPERATION, 12345) == pls.STATUS_INPUT_PARAMETER_ERROR
    assert A.hint(9999, pls.OPERATION_NOTRANS) == pls.STATUS_INPUT_PARAMETER_ERROR
    A.print_err()
    B = pls.SpMat.bsr(91, 4, 4, 3, np.array([0, 0]), np.zeros(0), np.zeros(0), check=False)
    assert B.status == pls.STATUS_INPUT_PARAMETER_ERROR
    assert A.update([0], [0], [2.0]) == 0
    assert A.update([0], [5], [2.0]) == pls.STATUS_INPUT_PARAMETER_ERROR


def test_special_handles():
    I = pls.SpMat.identity(4)
    np.testing.assert_array_equal(I.spmv(np.arange(4.0), np.ones(4), alpha=2.0, beta=1.0), 2 * np.arange(4.0) + 1)
    N = pls.SpMat.null(3, 2)
    np.testing.assert_array_equal(N.spmv(np.ones(2), np.array([1.0, 2.0, 3.0]), beta=-1.0), [-1.0, -2.0, -3.0])
    D = pls.SpMat.dense(pls.ROW_MAJOR, 2, 3, 3, np.arange(6.0))
    np.testing.assert_allclose(D.spmv(np.ones(3)), [3.0, 12.0])
    np.testing.assert_allclose(D.spmv(np.ones(2), trans=pls.OPERATION_TRANS), [3.0, 5.0, 7.0])


def test_transpose_ops():
    rng = np.random.default_rng(8)
    rp, c, v = W.random_csr(400, 300, 30, rng)
    x = rng.uniform(-1, 1, 400)
    y0 = rng.uniform(-1, 1, 300)
    yref = oracle.csr_spmv_trans(rp, c, v, 300, x, y=y0, alpha=1.25, beta=0.5)
    A = pls.SpMat.csr(400, 300, rp, c, v)
    y = A.spmv(x, y0.copy(), alpha=1.25, beta=0.5, trans=pls.OPERATION_TRANS)
    np.testing.assert_allclose(y, yref, rtol=1e-11, atol=1e-12)
    # optimized for the transpose (CSR of A^T)
    A = pls.SpMat.csr(400, 300, rp, c, v)
    A.hint(pls.HINT_SPMV_OPERATION, pls.OPERATION_TRANS)
    assert A.optimize() == 0
    y = A.spmv(x, y0.copy(), alpha=1.25, beta=0.5, trans=pls.OPERATION_TRANS)
    np.testing.assert_allclose(y, yref, rtol=1e-11, atol=1e-12)
    # and back to NOTRANS
    xr = rng.uniform(-1, 1, 300)
    np.testing.assert_allclose(A.spmv(xr), oracle.csr_spmv(rp, c, v, xr), rtol=1e-12, atol=1e-13)
    # values updated after the CSR of A^T was built: the transpose sees them
    rows = np.repeat(np.arange(400), np.diff(rp))[::7].astype(np.int32)
    cols = c[::7].astype(np.int32)
    assert A.update(rows, cols, np.full(len(rows), 3.0)) == 0
    v2 = v.copy()
    v2[::7] = 3.0
    yref2 = oracle.csr_spmv_trans(rp, c, v2, 300, x, y=y0, alpha=1.25, beta=0.5)
    y = A.spmv(x, y0.copy(), alpha=1.25, beta=0.5, trans=pls.OPERATION_TRANS)
    np.testing.assert_allclose(y, yref2, rtol=1e-11, atol=1e-12)


def test_device_pointer_exec_on_torch_stream():
    import torch

    rng = np.random.default_rng(4)
    rp, c, v = W.random_csr(3000, 2000, 50, rng)
    x = rng.uniform(-1, 1, 2000)
    A = pls.SpMat.csr(3000, 2000, rp, c, v)
    A.force_config(pls.KIND_SELL, 32, 256, 0)
    assert A.optimize() == 0
    xd = torch.tensor(x, device="cuda")
    yd = torch.full((3000,), float("nan"), dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        A.spmv_dev(xd.data_ptr(), yd.data_ptr(), 1.0, 0.0, s.cuda_stream)
    s.synchronize()
    yref = oracle.csr_spmv(rp, c, v, x)
    assert rel_err_rows(yd.cpu().numpy(), yref, scale_of(rp, c, v, x, 1, 0, None)).max() <= FP64_TOL


@pytest.fixture(scope="module")
def zipf_large():
    m, n, rp, c, v = W.zipf_rows(2_500_011, seed=21)
    rng = np.random.default_rng(22)
    return m, n, rp, c, v, W.uniform_vector(n, 23), rng.uniform(-1, 1, m)


@pytest.mark.parametrize("cfg", [(pls.KIND_SELL, 32, 4096, 0), (pls.KIND_SELL, 16, 48, 0),
                                 (pls.KIND_SELL, 8, 0, 0), (pls.KIND_CSR, 0, 0, 4),
                                 (pls.KIND_CSR_SPLIT, 0, 0, 256)])
def test_host_exec_in_row_bands(zipf_large, cfg):
    """Host-buffer calls with a y of 20 MB run in row bands, each band's rows
    copied back while the next computes. Without bands the host call is the
    device path bit for bit; with them, rows of chunks the band plan slices
    more finely are summed in another order, within the FP64 tolerance."""
    import torch

    m, n, rp, c, v, x, y0 = zipf_large
    A = pls.SpMat.csr(m, n, rp, c, v)
    assert A.force_config(*cfg) == 0
    assert A.optimize() == 0
    for alpha, beta in ((1.0, 0.0), (-0.75, 1.5)):
        yref = oracle.csr_spmv(rp, c, v, x, y=y0, alpha=alpha, beta=beta)
        sc = scale_of(rp, c, v, x, alpha, beta, y0)
        A.set_host_bands(0)
        yb = A.spmv(x, y0.copy(), alpha=alpha, beta=beta)
        assert A.host_bands_used() == 4, cfg
        assert rel_err_rows(yb, yref, sc).max() <= FP64_TOL
        A.set_host_bands(1)
        y1 = A.spmv(x, y0.copy(), alpha=alpha, beta=beta)
        assert A.host_bands_used() == 0
        xd = torch.tensor(x, device="cuda")
        yd = torch.tensor(y0, device="cuda")
        torch.cuda.synchronize()
        A.spmv_dev(xd.data_ptr(), yd.data_ptr(), alpha, beta)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(y1, yd.cpu().numpy())
        for nb in (2, 7, 64):
            A.set_host_bands(nb)
            y = A.spmv(x, y0.copy(), alpha=alpha, beta=beta)
            assert 2 <= A.host_bands_used() <= nb
            assert rel_err_rows(y, yref, sc).max() <= FP64_TOL, (cfg, nb)
    A.destroy()


def test_host_exec_in_row_bands_fp32():
    m, n, rp, c, v = W.zipf_rows(2_200_003, seed=24)
    x = W.uniform_vector(n, 25).astype(np.float32)
    A = pls.SpMat.csr(m, n, rp, c, v.astype(np.float32))
    assert A.force_config(pls.KIND_SELL, 32, 1024, 0) == 0
    assert A.optimize() == 0
    y = A.spmv(x)
    yref = oracle.csr_spmv(rp, c, v, x.astype(np.float64))
    sc = scale_of(rp, c, v, x.astype(np.float64), 1.0, 0.0, None)
    assert rel_err_rows(y.astype(np.float64), yref, sc).max() <= 1e-5
    A.destroy()


# ------------------------------------------------------- reduced precision


@pytest.mark.parametrize("storage,tol", [(pls.STORAGE_FP32, 1e-5), (pls.STORAGE_BF16, 1e-2)])
def test_reduced_storage_error(storage, tol):
    m, n, rp, c, v = W.zipf_rows(50_000, seed=21)
    x = W.uniform_vector(n, 22)
    yref = oracle.csr_spmv(rp, c, v, x)
    sc = scale_of(rp, c, v, x, 1, 0, None)
    for cfg in [(pls.KIND_CSR, 0, 0, 8), (pls.KIND_SELL, 32, 1024, 0)]:
        y = gpu_spmv(rp, c, v, m, n, x, None, 1.0, 0.0, cfg, storage=storage)
        err = rel_err_rows(y, yref, sc).max()
        assert err <= tol, (storage, cfg, err)
    # float API with bf16 storage
    A = pls.SpMat.csr(m, n, rp, c, v.astype(np.float32))
    A.set_storage(storage)
    A.optimize()
    yf = A.spmv(x.astype(np.float32))
    assert rel_err_rows(yf.astype(np.float64), yref, sc).max() <= max(tol, 1e-5)
