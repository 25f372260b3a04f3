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


@pytest.mark.parametrize("C_,sigma", [(32, 4096), (16, 16384), (8, 0)])
def test_noalloc_matches_device_entry_point_twice(C_, sigma):
    import torch

    # Power-law rows: the widest chunks are sliced, so the partial sums go
    # through the fixed scratch array.
    m, n, rp, c, v = W.zipf_rows(200_000, seed=11)
    x = W.uniform_vector(n, 12)
    y0 = W.uniform_vector(m, 13)
    A = pls.SpMat.csr(m, n, rp, c, v)
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
        assert _scaled_err(y, y_existing, rp, c, v, x, alpha, beta, y0) <= TOL, call
    # and both agree with the oracle
    y_oracle = oracle.csr_spmv(rp, c, v, x, y=y0, alpha=alpha, beta=beta)
    assert _scaled_err(y, y_oracle, rp, c, v, x, alpha, beta, y0) <= TOL


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
