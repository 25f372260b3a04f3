"""GPU: sizes far past 32-bit byte offsets. 2^30 stored entries (an 8 GiB
value array, a 4 GiB column array, 2^25 rows) through the CSR kernel, the
SELL-C-sigma layout and kernel, the host-buffer path in row bands and the
SpMM kernels. Values are 1 and x / B hold small integers, so every result is
an integer below 2^53 and must be exact in any summation order: the check is
equality with a sum computed by torch. About 45 GB of device memory at the
peak."""
import numpy as np
import pytest

import perf_libs_sparse_b200 as pls

pytestmark = pytest.mark.gpu

M = 1 << 25       # rows (= columns)
W = 32            # entries per row
CHUNK = 1 << 26   # entries generated per step


def test_billion_entries_exact():
    import torch

    dev = "cuda"
    nnz = M * W
    rp = (torch.arange(M + 1, dtype=torch.int64, device=dev) * W).to(torch.int32)
    col = torch.empty(nnz, dtype=torch.int32, device=dev)
    for j0 in range(0, nnz, CHUNK):
        j = torch.arange(j0, min(nnz, j0 + CHUNK), dtype=torch.int64, device=dev)
        col[j0:j0 + len(j)] = ((j * 2654435761) % M).to(torch.int32)  # Knuth's multiplicative hash
        del j
    vals = torch.ones(nnz, dtype=torch.float64, device=dev)
    # y_ref[i] = sum of row i's columns (x = column index)
    y_ref = torch.empty(M, dtype=torch.float64, device=dev)
    rows_per = CHUNK // W
    for r0 in range(0, M, rows_per):
        y_ref[r0:r0 + rows_per] = col[r0 * W:(r0 + rows_per) * W].view(-1, W).to(torch.float64).sum(1)
    torch.cuda.synchronize()
    A = pls.SpMat.csr_dev(M, M, rp.data_ptr(), col.data_ptr(), vals.data_ptr())
    del vals
    torch.cuda.empty_cache()
    x = torch.arange(M, dtype=torch.float64, device=dev)
    y = torch.empty(M, dtype=torch.float64, device=dev)
    for cfg in [(pls.KIND_CSR, 0, 0, 8), (pls.KIND_SELL, 32, 0, 0), (pls.KIND_SELL, 16, 4096, 0)]:
        assert A.force_config(*cfg) == 0
        assert A.optimize() == 0
        y.fill_(float("nan"))
        torch.cuda.synchronize()
        A.spmv_dev(x.data_ptr(), y.data_ptr(), 1.0, 0.0)
        torch.cuda.synchronize()
        assert torch.equal(y, y_ref), cfg
    # host buffers, row bands (a 256 MiB result: 8 bands)
    yh = A.spmv(x.cpu().numpy())
    assert A.host_bands_used() == 8
    assert np.array_equal(yh, y_ref.cpu().numpy())
    del y
    # SpMM, k = 8: B[c, j] = c * (j + 1), so C[i, j] = y_ref[i] * (j + 1)
    k = 8
    scale = torch.arange(1, k + 1, dtype=torch.float64, device=dev)
    B = x[:, None] * scale[None, :]
    Cm = torch.empty((M, k), dtype=torch.float64, device=dev)
    for path in (-1, 2):
        A.set_spmm_path(path)
        Cm.fill_(float("nan"))
        torch.cuda.synchronize()
        A.spmm_dev(B.data_ptr(), k, k, Cm.data_ptr(), k, 1.0, 0.0)
        torch.cuda.synchronize()
        assert torch.equal(Cm, y_ref[:, None] * scale[None, :]), path
    A.destroy()
    del B, Cm, x, col, rp, y_ref
    torch.cuda.empty_cache()
