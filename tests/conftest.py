import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def guard_build_check():
    """Under the guard build of the library (PERFLIBS_B200_LIBRARY naming
    libplsparse_b200_guard.so), the session fails if any kernel wrote past a
    device buffer's end. The handles still alive are freed first, since the
    guards are checked when buffers are freed."""
    yield
    if os.environ.get("PERFLIBS_B200_LIBRARY", "").endswith("_guard.so"):
        import gc

        import perf_libs_sparse_b200 as pls

        gc.collect()
        assert pls.debug_guard_violations() == 0


@pytest.fixture(scope="session")
def kats():
    with open(os.path.join(GOLDEN, "reference_kats.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def ref_outputs():
    return np.load(os.path.join(GOLDEN, "ref_outputs.npz"))


def case_names(npz):
    return sorted({k.split("/")[0] for k in npz.files})


def rel_err_rows(y, y_ref, scale):
    """Per-row error |y - y_ref| / max(|y_ref|, scale_i): the row scale is
    |alpha| * sum_j |a_ij x_j| + |beta| |y0_i|, the magnitude a summation-order
    change can perturb, so cancelling rows are measured fairly."""
    den = np.maximum(np.abs(y_ref), scale)
    den = np.where(den == 0, 1.0, den)
    return np.abs(y - y_ref) / den


@pytest.fixture(scope="session")
def ref_spmm():
    return np.load(os.path.join(GOLDEN, "ref_spmm.npz"))


def spmm_case_csr(f, name):
    """A fixture case as 0-based CSR (BSR cases through the oracle's
    bsr2csr, which keeps the reference's CSR view: explicit zeros dropped)."""
    import oracle

    if int(f[f"{name}/kind"]) == 1:
        return oracle.bsr2csr(f[f"{name}/row_ptr"], f[f"{name}/col"], f[f"{name}/vals"],
                              int(f[f"{name}/bs"]), int(f[f"{name}/layout"]))
    base = int(f[f"{name}/base"])
    return ((f[f"{name}/row_ptr"] - base).astype(np.int32), (f[f"{name}/col"] - base).astype(np.int32),
            f[f"{name}/vals"])


def spmm_row_err(got, ref, rp, col, vals, B, alpha, beta=0.0, C0=None):
    """Per-row scaled error of an SpMM result: |got - ref| over
    max(|ref|, |alpha| sum_j |a_ij| |B_j| + |beta| |C0|), elementwise."""
    import oracle

    k = B.shape[1]
    scale = abs(alpha) * oracle.csr_spmm(rp, col, np.abs(vals), np.abs(B), k)
    if C0 is not None:
        scale = scale + abs(beta) * np.abs(C0)
    den = np.maximum(np.abs(ref), scale)
    den = np.where(den == 0, 1.0, den)
    return float((np.abs(got - ref) / den).max())
