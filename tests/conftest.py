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
    change can perturb, so cancelling rows are judged fairly."""
    den = np.maximum(np.abs(y_ref), scale)
    den = np.where(den == 0, 1.0, den)
    return np.abs(y - y_ref) / den
