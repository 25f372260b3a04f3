"""GPU: the allocation-free SpMV entry point (perflibs_b200_spmv_exec_d_noalloc).

It exists for callers that cannot call cudaMalloc around their SpMV — code
whose device memory belongs to a pool or caching allocator of its own, and
latency-critical loops where an allocation's device synchronisation is not
acceptable. Its partial sums live in one fixed device array, so this test
checks it through the C-ABI against the existing device-pointer entry point
(perflibs_b200_spmv_exec_d_dev) on two calls in a row: the second call
starts from the first call's leftovers in the shared array and must give
the same result. The file name sorts last so that a run stopping at the
first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
import perf_libs_sparse_b200 as pls
from perf_libs_sparse_b200 import workloads as W
from tests.conftest import rel_err_rows

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the FP64 parity tolerance used by every SpMV test


def _noalloc():
    fn = pls.lib().perflibs_b200_spmv_exec_d_noalloc
    fn.argtypes = [C.c_double, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    return fn


def _scaled_err(y, y_ref, rp, c, v, x, alpha, beta, y0):
    scale = abs(alpha) * oracle.csr_absdot(rp, c, v, x) + abs(beta) * np.abs(y0)
    return rel_err_rows(y, y_ref, scale).max()


@pytest.mark.parametrize("C_,sigma,storage", [(32, 4096, pls.STORAGE_NATIVE), (16, 8192, pls.STORAGE_NATIVE),
                                               (8, 0, pls.STORAGE_NATIVE), (32, 4096, pls.STORAGE_FP32),
                                               (16, 1024, pls.STORAGE_BF16)])
def test_noalloc_matches_device_entry_point_twice(C_, sigma, storage):
    import torch

    # Power-law rows: the widest chunks are sliced, so the partial sums go
    # through the fixed scratch array. With FP32 / BF16 value storage the
    # slices' FP32 partial sums share the same array.
    m, n, rp, c, v = W.zipf_rows(200_000, seed=11)
    x = W.uniform_vector(n, 12)
    y0 = W.uniform_vector(m, 13)
    A = pls.SpMat.csr(m, n, rp, c, v)
    A.set_storage(storage)
    assert A.force_config(pls.KIND_SELL, C_, sigma, 0) == 0
    assert A.optimize() == 0
    assert A.config()["kind"] == pls.KIND_SELL
    if sigma == 4096:
        assert A.exec_info()["n_split"] > 0  # the scratch really is used

    stream = torch.cuda.Stream()
    xd = torch.tensor(x, device="cuda")
    alpha, beta = 1.25, -0.5
    y_ref_dev = torch.tensor(y0, device="cuda")
    A.spmv_dev(xd.data_ptr(), y_ref_dev.data_ptr(), alpha, beta, stream.cuda_stream)
    stream.synchronize()
    y_existing = y_ref_dev.cpu().numpy()

    fn = _noalloc()
    for call in range(2):
        yd = torch.tensor(y0, device="cuda")
        st = fn(alpha, A.h, C.c_void_p(xd.data_ptr()), beta, C.c_void_p(yd.data_ptr()),
                C.c_void_p(stream.cuda_stream))
        assert st == pls.STATUS_SUCCESS, call
        stream.synchronize()
        y = yd.cpu().numpy()
        # the same kernel over the same work list: the same bits
        np.testing.assert_array_equal(y, y_existing, err_msg=f"call {call}")
    # and both agree with the oracle, within the storage mode's tolerance
    y_oracle = oracle.csr_spmv(rp, c, v, x, y=y0, alpha=alpha, beta=beta)
    tol = {pls.STORAGE_NATIVE: TOL, pls.STORAGE_FP32: 1e-5, pls.STORAGE_BF16: 1e-2}[storage]
    assert _scaled_err(y, y_oracle, rp, c, v, x, alpha, beta, y0) <= tol


def test_noalloc_rejects_handles_without_sell_layout():
    import torch

    rng = np.random.default_rng(1)
    rp, c, v = W.random_csr(100, 100, 10, rng)
    A = pls.SpMat.csr(100, 100, rp, c, v)
    A.force_config(pls.KIND_CSR, 0, 0, 4)
    assert A.optimize() == 0
    xd = torch.zeros(100, dtype=torch.float64, device="cuda")
    yd = torch.zeros(100, dtype=torch.float64, device="cuda")
    st = _noalloc()(1.0, A.h, C.c_void_p(xd.data_ptr()), 0.0, C.c_void_p(yd.data_ptr()), None)
    assert st == pls.STATUS_INPUT_PARAMETER_ERROR


def test_noalloc_rejects_a_matrix_beyond_the_fixed_scratch():
    """A layout whose column slices need more partial sums than the fixed
    array holds (2^21 elements) is refused with an input error naming both
    sizes, and y is left untouched; the device-pointer entry point, which
    allocates its own scratch, still runs it. 450,000 chunks of 32 rows:
    every 20th holds one row of 200 entries (3 slices of 81 columns each),
    and one row has 4096 entries, so the slices need 67,551 x 32 partial
    sums."""
    import torch

    nC, C_ = 450_000, 32
    m, n = nC * C_, 8192
    lens = np.zeros(m, np.int64)
    lens[np.arange(0, nC, 20) * C_] = 200
    lens[1 * C_] = 4096
    rp = np.zeros(m + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    nnz = int(rp[-1])
    starts = np.repeat(rp[:-1].astype(np.int64), lens)
    col = (np.arange(nnz, dtype=np.int64) - starts).astype(np.int32)  # columns 0 .. len-1
    v = np.random.default_rng(3).uniform(-1, 1, nnz)
    A = pls.SpMat.csr(m, n, rp, col, v)
    assert A.force_config(pls.KIND_SELL, C_, 0, 0) == 0
    assert A.optimize() == 0
    info = A.exec_info()
    assert info["n_items"] * C_ > 2 ** 21, info
    xd = torch.tensor(W.uniform_vector(n, 4), device="cuda")
    yd = torch.full((m,), 7.0, dtype=torch.float64, device="cuda")
    st = _noalloc()(1.0, A.h, C.c_void_p(xd.data_ptr()), 0.0, C.c_void_p(yd.data_ptr()), None)
    torch.cuda.synchronize()
    assert st == pls.STATUS_INPUT_PARAMETER_ERROR
    msg = A.error()[2]
    assert str(info["n_items"] * C_) in msg and str(2 ** 21) in msg, msg
    assert bool((yd == 7.0).all())
    A.spmv_dev(xd.data_ptr(), yd.data_ptr(), 1.0, 0.0)
    torch.cuda.synchronize()
    rows = np.flatnonzero(lens)
    y = yd.cpu().numpy()
    x = xd.cpu().numpy()
    for r in rows[:50]:
        ref = float(np.dot(v[rp[r]:rp[r + 1]], x[:lens[r]]))
        assert abs(y[r] - ref) <= 1e-12 * max(1.0, float(np.abs(v[rp[r]:rp[r + 1]]).dot(np.abs(x[:lens[r]]))))
    assert np.all(y[lens == 0] == 0)
