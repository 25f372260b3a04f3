"""GPU parity at the full sizes of the benchmark configurations.

Each configuration is built with its stated generator and seed and run
through the C-ABI; results are checked against the FP64 oracle with the
per-row scaled error (|y - y_ref| / max(|y_ref|, sum_j |a_ij x_j|)):
1e-12 for FP64, 1e-5 for FP32 value storage, 1e-2 for BF16 value storage.

* C1: plain FP64 CSR SpMV and the tuned SpMV on the 5-point Laplacian 512^2,
  every row.
* C2: the tuned SELL-C-sigma SpMV and the plain CSR kernel on the power-law
  matrix (n = 4,194,304), every row.
* C3: CSR SpMM on the 27-point 128^3 stencil, k in {8, 32, 128}, FP64 /
  FP32 / BF16 value storage, every SpMM kernel forced once besides the
  measured choice. All rows for k <= 32; for k = 128 (a 2.1 GB result)
  8 blocks of 16384 rows spread over the matrix, the first and last
  included.
* C4: all 512 instances of the uneven batch (FP32), tuned, with and
  without the staged items, every row of every instance.
"""
import numpy as np
import pytest

import oracle
import perf_libs_sparse_b200 as pls
from perf_libs_sparse_b200 import workloads as W
from tests.conftest import rel_err_rows

pytestmark = pytest.mark.gpu

TOLS = {"native": 1e-12, "fp32": 1e-5, "bf16": 1e-2}
STORAGE = {"native": pls.STORAGE_NATIVE, "fp32": pls.STORAGE_FP32, "bf16": pls.STORAGE_BF16}
# SpMM kernels: -1 measured choice, 0 row group, 1 staged, 2 row group with
# shared entries, 3 diagonal form, 4 diagonal form with TMA-staged B.
SPMM_PATHS = (-1, 0, 1, 2, 3, 4)


def _spmv_err(y, rp, c, v, x):
    y_ref = oracle.csr_spmv(rp, c, v, x)
    return rel_err_rows(y, y_ref, oracle.csr_absdot(rp, c, v, x)).max()


def _run_spmv(A, x, m):
    import torch

    xd = torch.tensor(x, device="cuda")
    yd = torch.full((m,), float("nan"), dtype=torch.float64, device="cuda")
    A.spmv_dev(xd.data_ptr(), yd.data_ptr(), 1.0, 0.0)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def test_c1_laplacian_full():
    m, n, rp, c, v = W.laplacian_2d(512)
    assert (m, int(rp[-1])) == (262_144, 1_308_672)
    x = W.uniform_vector(n, 0)
    for inv in (pls.INVOCATIONS_SINGLE, pls.INVOCATIONS_MANY):  # plain CSR, then tuned
        A = pls.SpMat.csr(m, n, rp, c, v)
        A.hint(pls.HINT_SPMV_INVOCATIONS, inv)
        assert A.optimize() == 0
        assert _spmv_err(_run_spmv(A, x, m), rp, c, v, x) <= 1e-12, inv
        # the drop-in host-buffer call too
        assert _spmv_err(A.spmv(x), rp, c, v, x) <= 1e-12, inv
        A.destroy()


def test_c2_powerlaw_full():
    m, n, rp, c, v = W.zipf_rows(4_194_304, seed=1)
    x = W.uniform_vector(n, 1)
    assert m == 4_194_304 and 60_000_000 < int(rp[-1]) < 75_000_000
    A = pls.SpMat.csr(m, n, rp, c, v)
    A.hint(pls.HINT_SPMV_INVOCATIONS, pls.INVOCATIONS_MANY)
    assert A.optimize() == 0
    cfg = A.config()
    if cfg["kind"] == pls.KIND_SELL:
        assert cfg["C"] in (8, 16, 32) and (cfg["sigma"] == 0 or 32 <= cfg["sigma"] <= 8192), cfg
    assert _spmv_err(_run_spmv(A, x, m), rp, c, v, x) <= 1e-12
    A.destroy()
    P = pls.SpMat.csr(m, n, rp, c, v)
    P.hint(pls.HINT_SPMV_INVOCATIONS, pls.INVOCATIONS_SINGLE)
    assert P.optimize() == 0
    assert _spmv_err(_run_spmv(P, x, m), rp, c, v, x) <= 1e-12
    P.destroy()


@pytest.fixture(scope="module")
def c3():
    m, n, rp, c, v = W.stencil_27pt(128, seed=2)
    assert (m, int(rp[-1])) == (2_097_152, 55_742_968)
    return m, n, rp, c, v


def _blocks(m, full):
    if full:
        return [(r, min(m, r + 262144)) for r in range(0, m, 262144)]
    starts = np.linspace(0, m - 16384, 8).astype(np.int64)
    return [(int(s), int(s) + 16384) for s in starts]


@pytest.fixture(scope="module")
def c3_refs(c3):
    """FP64 oracle results (and row scales) of C3 per k on the checked row
    blocks, computed once: {k: (B, [(r0, r1, ref, scale)])}."""
    m, n, rp, c, v = c3
    Bfull = np.random.default_rng(2).uniform(-1, 1, (n, 128))
    out = {}
    for k in (8, 32, 128):
        B = np.ascontiguousarray(Bfull[:, :k])
        blocks = []
        for r0, r1 in _blocks(m, k <= 32):
            p0, p1 = int(rp[r0]), int(rp[r1])
            sub = (rp[r0:r1 + 1] - rp[r0]).astype(np.int32)
            ref = oracle.csr_spmm(sub, c[p0:p1], v[p0:p1], B, k)
            scale = oracle.csr_spmm(sub, c[p0:p1], np.abs(v[p0:p1]), np.abs(B), k)
            blocks.append((r0, r1, ref, scale))
        out[k] = (B, blocks)
    return out


@pytest.mark.parametrize("k", [8, 32, 128])
@pytest.mark.parametrize("storage", ["native", "fp32", "bf16"])
def test_c3_stencil_spmm_full(c3, c3_refs, k, storage):
    import torch

    m, n, rp, c, v = c3
    B, blocks = c3_refs[k]
    native = storage == "native"
    dt = np.float64 if native else np.float32
    tdt = torch.float64 if native else torch.float32
    A = pls.SpMat.csr(m, n, rp, c, v.astype(dt))
    A.set_storage(STORAGE[storage])
    assert A.optimize() == 0
    Bd = torch.tensor(B, dtype=tdt, device="cuda")
    Cd = torch.empty((m, k), dtype=tdt, device="cuda")
    ran = set()
    for path in SPMM_PATHS:
        A.set_spmm_path(path)
        Cd.fill_(float("nan"))
        A.spmm_dev(Bd.data_ptr(), k, k, Cd.data_ptr(), k, 1.0, 0.0)
        torch.cuda.synchronize()
        ran.add(A.spmm_info()["path"])
        worst = 0.0
        for r0, r1, ref, scale in blocks:
            got = Cd[r0:r1].cpu().numpy().astype(np.float64)
            den = np.maximum(np.abs(ref), scale)
            den[den == 0] = 1
            worst = max(worst, float((np.abs(got - ref) / den).max()))
        assert worst <= TOLS[storage], (k, storage, path, worst)
    # the row group, shared entries, diagonal and TMA-staged diagonal
    # kernels each ran once, and the staged kernel with FP64 / FP32 values
    assert {0, 2, 3, 4} <= ran, ran
    if storage != "bf16":
        assert 1 in ran, ran
    A.destroy()


@pytest.fixture(scope="module")
def c4():
    return W.batched_instances(512, seed=3)


def test_c4_batch_full(c4):
    import torch

    inst = c4
    mats, Bs, Cs = [], [], []
    for d in inst:
        if d["kind"] == "bsr":
            mats.append(pls.SpMat.bsr(d["layout"], d["m"], d["n"], d["bs"], d["row_ptr"], d["col"], d["vals"]))
        else:
            mats.append(pls.SpMat.csr(d["m"], d["n"], d["row_ptr"], d["col"], d["vals"]))
        Bs.append(torch.tensor(d["B"], device="cuda"))
        Cs.append(torch.full((d["m"], d["k"]), float("nan"), dtype=torch.float32, device="cuda"))
    ks = [d["k"] for d in inst]
    bt = pls.Batch(mats, ks, [b.data_ptr() for b in Bs], ks, [c_.data_ptr() for c_ in Cs], ks)
    bt.tune()
    refs = []
    for d in inst:
        if d["kind"] == "bsr":
            rp, cc, vv = oracle.bsr2csr(d["row_ptr"], d["col"], d["vals"].astype(np.float64), d["bs"], d["layout"])
        else:
            rp, cc, vv = d["row_ptr"], d["col"], d["vals"].astype(np.float64)
        B = d["B"].astype(np.float64)
        ref = oracle.csr_spmm(rp, cc, vv, B, d["k"])
        scale = oracle.csr_spmm(rp, cc, np.abs(vv), np.abs(B), d["k"])
        refs.append((ref, scale))
    for staging in (True, False):
        bt.set_staging(staging)
        for Cd in Cs:
            Cd.fill_(float("nan"))
        bt.exec(1.0, 0.0)
        torch.cuda.synchronize()
        for i, (Cd, (ref, scale)) in enumerate(zip(Cs, refs)):
            got = Cd.cpu().numpy().astype(np.float64)
            den = np.maximum(np.abs(ref), scale)
            den[den == 0] = 1
            err = float((np.abs(got - ref) / den).max()) if got.size else 0.0
            assert err <= 1e-5, (i, inst[i]["kind"], staging, err)
    bt.destroy()
    for A in mats:
        A.destroy()
