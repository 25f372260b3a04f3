"""GPU: the batched uneven SpMM (one persistent launch in a CUDA graph)
against the oracle, per instance. FP32 values and accumulation: per-element
error scaled by |alpha| sum_j |a_ij b_jk| + |beta| |c0| must stay <= 1e-5."""
import numpy as np
import pytest

import oracle
import perf_libs_sparse_b200 as pls
from perf_libs_sparse_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _reference(d, alpha, beta, C0):
    if d["kind"] == "bsr":
        rp, c, v = oracle.bsr2csr(d["row_ptr"], d["col"], d["vals"].astype(np.float64), d["bs"], d["layout"])
    else:
        rp, c, v = d["row_ptr"], d["col"], d["vals"].astype(np.float64)
    B = d["B"].astype(np.float64)
    ref = oracle.csr_spmm(rp, c, v, B, d["k"], Cmat=C0.astype(np.float64), alpha=alpha, beta=beta)
    scale = abs(alpha) * oracle.csr_spmm(rp, c, np.abs(v), np.abs(B), d["k"]) + abs(beta) * np.abs(C0)
    return ref, scale


@pytest.mark.parametrize("tile", [0, 8, 2048])
def test_batch_matches_oracle(tile):
    import torch

    inst = W.batched_instances(count=36, seed=3, n_lo=256, n_hi=4096)
    mats, Bs, Cs, C0s = [], [], [], []
    rng = np.random.default_rng(0)
    for d in inst:
        if d["kind"] == "bsr":
            mats.append(pls.SpMat.bsr(d["layout"], d["m"], d["n"], d["bs"], d["row_ptr"], d["col"], d["vals"]))
        else:
            mats.append(pls.SpMat.csr(d["m"], d["n"], d["row_ptr"], d["col"], d["vals"]))
        Bs.append(torch.tensor(d["B"], device="cuda"))
        c0 = rng.uniform(-1, 1, (d["m"], d["k"])).astype(np.float32)
        C0s.append(c0)
        Cs.append(torch.tensor(c0, device="cuda"))
    s = torch.cuda.Stream()
    bt = pls.Batch(mats, [d["k"] for d in inst], [b.data_ptr() for b in Bs], [d["k"] for d in inst],
                   [c.data_ptr() for c in Cs], [d["k"] for d in inst], stream=s.cuda_stream)
    if tile == 0:
        best, ms = bt.tune()
        assert best > 0 and ms > 0
        for c, c0 in zip(Cs, C0s):  # tuning ran with beta = 0: restore C0
            c.copy_(torch.tensor(c0, device="cuda"))
        torch.cuda.synchronize()
    else:
        bt.set_tile(tile)
    assert bt.info()["launches"] == 1
    bt.exec(1.5, 0.5)
    s.synchronize()
    for d, c, c0 in zip(inst, Cs, C0s):
        ref, scale = _reference(d, 1.5, 0.5, c0)
        got = c.cpu().numpy().astype(np.float64)
        den = np.maximum(np.abs(ref), scale)
        den[den == 0] = 1
        assert (np.abs(got - ref) / den).max() <= 1e-5, (d["kind"], d["m"], d["k"])
    # a second exec with beta = 0 overwrites
    bt.exec(1.0, 0.0)
    s.synchronize()
    for d, c in zip(inst, Cs):
        ref, scale = _reference(d, 1.0, 0.0, np.zeros((d["m"], d["k"])))
        got = c.cpu().numpy().astype(np.float64)
        den = np.maximum(np.abs(ref), scale)
        den[den == 0] = 1
        assert (np.abs(got - ref) / den).max() <= 1e-5
