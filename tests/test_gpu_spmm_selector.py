"""GPU: the learned SpMM kernel selectors attached to a handle
(perflibs_b200_spmat_set_spmm_selectors). With a selector attached for the
call's k, the first SpMM of a signature runs a predicted kernel without
timing the candidates (spmm_info reports no timings) and the result still
matches the oracle; a selector with the wrong number of classes is refused;
detaching brings the measured choice back."""
import numpy as np
import pytest

import oracle
import perf_libs_sparse_b200 as pls
from perf_libs_sparse_b200 import selector as S
from perf_libs_sparse_b200 import workloads as W
from tests.conftest import spmm_row_err

pytestmark = pytest.mark.gpu


def _spmm(A, Bd, k, m):
    import torch

    Bt = torch.tensor(Bd, device="cuda")
    Ct = torch.full((m, k), float("nan"), dtype=torch.float64, device="cuda")
    A.spmm_dev(Bt.data_ptr(), k, k, Ct.data_ptr(), k, 1.0, 0.0)
    torch.cuda.synchronize()
    return Ct.cpu().numpy()


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_predicted_kernel_runs_untimed_and_matches_oracle(seed):
    rng = np.random.default_rng(seed)
    sels = S.default_spmm_selectors() or [S.Selector(len(S.SPMM_CLASSES), seed=seed + b) for b in range(3)]
    for (m, n, rp, c, v) in (W.stencil_27pt(20, seed=2), W.banded_csr(6000, 9, rng)):
        A = pls.SpMat.csr(m, n, rp, c, v)
        S.attach_spmm_selectors(A, sels)
        for k in (8, 32, 128):
            Bd = rng.uniform(-1, 1, (n, k))
            got = _spmm(A, Bd, k, m)
            info = A.spmm_info()
            assert info["ms_rows"] == 0 and info["ms_staged"] == 0, info  # nothing was timed
            assert info["path"] in (0, 1, 2, 3, 4), info
            ref = oracle.csr_spmm(rp, c, v, Bd, k)
            assert spmm_row_err(got, ref, rp, c, v, Bd, 1.0) <= 1e-12, (k, info)
        # detached: the next signature is measured again
        S.attach_spmm_selectors(A, None)
        k = 16
        Bd = rng.uniform(-1, 1, (n, k))
        got = _spmm(A, Bd, k, m)
        assert A.spmm_info()["ms_rows"] > 0
        assert spmm_row_err(got, oracle.csr_spmm(rp, c, v, Bd, k), rp, c, v, Bd, 1.0) <= 1e-12
        A.destroy()


def test_selector_with_wrong_class_count_is_refused():
    rp, c, v = W.random_csr(50, 50, 5, np.random.default_rng(3))
    A = pls.SpMat.csr(50, 50, rp, c, v)
    wrong = S.Selector(7)
    with pytest.raises(pls.PerflibsError) as e:
        S.attach_spmm_selectors(A, [wrong, None, None])
    assert e.value.status == pls.STATUS_INPUT_PARAMETER_ERROR
