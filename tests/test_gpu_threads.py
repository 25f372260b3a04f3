"""GPU: handles used from several host threads at once. Calls on distinct
handles are independent (the reference's rule; a handle itself is not
thread-safe): four threads each create, tune and run their own matrix
through the host-buffer and device-pointer entry points while the others
do the same, and every result matches the oracle. ctypes releases the GIL
for the duration of each library call, so the calls really overlap."""
import threading

import numpy as np
import pytest

import oracle
import perf_libs_sparse_b200 as pls
from perf_libs_sparse_b200 import workloads as W
from tests.conftest import rel_err_rows

pytestmark = pytest.mark.gpu


def _worker(seed, errors):
    import torch

    try:
        rng = np.random.default_rng(seed)
        if seed % 2:
            m, n, rp, c, v = W.zipf_rows(300_000 + 1000 * seed, seed=seed)
        else:
            m = n = 200_000 + 1000 * seed
            rp, c, v = W.random_csr(m, n, 40, rng)
        x = rng.uniform(-1, 1, n)
        y0 = rng.uniform(-1, 1, m)
        A = pls.SpMat.csr(m, n, rp, c, v)
        assert A.optimize() == 0
        yref = oracle.csr_spmv(rp, c, v, x, y=y0, alpha=1.5, beta=-0.25)
        sc = 1.5 * oracle.csr_absdot(rp, c, v, x) + 0.25 * np.abs(y0)
        s = torch.cuda.Stream()
        xd = torch.tensor(x, device="cuda")
        for _ in range(5):
            y = A.spmv(x, y0.copy(), alpha=1.5, beta=-0.25)
            assert rel_err_rows(y, yref, sc).max() <= 1e-12
            yd = torch.tensor(y0, device="cuda")
            torch.cuda.synchronize()
            A.spmv_dev(xd.data_ptr(), yd.data_ptr(), 1.5, -0.25, s.cuda_stream)
            s.synchronize()
            assert rel_err_rows(yd.cpu().numpy(), yref, sc).max() <= 1e-12
        A.destroy()
    except Exception as e:  # reported to the main thread
        errors.append((seed, repr(e)))


def test_four_threads_four_handles():
    import torch

    torch.cuda.init()
    errors = []
    threads = [threading.Thread(target=_worker, args=(seed, errors)) for seed in (1, 2, 3, 4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=600)
    assert not any(t.is_alive() for t in threads)
    assert not errors, errors
