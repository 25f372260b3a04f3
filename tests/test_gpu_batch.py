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


def test_batch_odd_blocks_layouts_and_values_at_creation():
    """BSR instances of block sizes 1, 2, 3 and 5 in both block layouts, with
    empty block rows; a CSR instance with empty rows; k from 1 to 13 with
    and without 16-byte vectors. The batch expands BSR instances into scalar
    rows at creation and reads its own copy of every instance's entries:
    values updated in a handle afterwards are seen once the batch is created
    again."""
    import torch

    rng = np.random.default_rng(9)
    mats, descs = [], []
    for bs, layout, k in [(1, pls.ROW_MAJOR, 3), (2, pls.COL_MAJOR, 8), (3, pls.ROW_MAJOR, 13),
                          (5, pls.COL_MAJOR, 4), (3, pls.COL_MAJOR, 1)]:
        mb, nb = 40, 30
        counts = rng.integers(0, 4, mb)
        counts[::7] = 0  # empty block rows
        rp = np.zeros(mb + 1, np.int32)
        rp[1:] = np.cumsum(counts)
        col = np.concatenate([np.sort(rng.choice(nb, c, replace=False)) for c in counts]).astype(np.int32)
        vals = rng.uniform(-1, 1, int(rp[-1]) * bs * bs).astype(np.float32)
        mats.append(pls.SpMat.bsr(layout, mb * bs, nb * bs, bs, rp, col, vals))
        descs.append(dict(kind="bsr", row_ptr=rp, col=col, vals=vals, bs=bs, layout=layout, m=mb * bs,
                          n=nb * bs, k=k))
    m, n = 700, 500
    rp, c, v = W.random_csr(m, n, 12, rng, empty_frac=0.3)
    v = v.astype(np.float32)
    mats.append(pls.SpMat.csr(m, n, rp, c, v))
    descs.append(dict(kind="csr", row_ptr=rp, col=c, vals=v, m=m, n=n, k=9))
    Bs, Cs = [], []
    for d in descs:
        d["B"] = rng.uniform(-1, 1, (d["n"], d["k"])).astype(np.float32)
        Bs.append(torch.tensor(d["B"], device="cuda"))
        Cs.append(torch.zeros((d["m"], d["k"]), dtype=torch.float32, device="cuda"))
    ks = [d["k"] for d in descs]
    s = torch.cuda.Stream()

    def run_and_check():
        bt = pls.Batch(mats, ks, [b.data_ptr() for b in Bs], ks, [c.data_ptr() for c in Cs], ks,
                       stream=s.cuda_stream)
        bt.set_tile(8)
        bt.exec(1.0, 0.0)
        s.synchronize()
        for d, cm in zip(descs, Cs):
            ref, scale = _reference(d, 1.0, 0.0, np.zeros((d["m"], d["k"])))
            got = cm.cpu().numpy().astype(np.float64)
            den = np.maximum(np.abs(ref), scale)
            den[den == 0] = 1
            assert (np.abs(got - ref) / den).max() <= 1e-5, (d["kind"], d.get("bs"), d["k"])
        return bt

    bt = run_and_check()
    # change the CSR instance's values: the existing batch keeps its copy
    rows = np.repeat(np.arange(m), np.diff(rp))[:5].astype(np.int32)
    cols = c[:5].astype(np.int32)
    assert mats[-1].update(rows, cols, np.full(5, 7.0, np.float32)) == 0
    descs[-1]["vals"] = v.copy()
    descs[-1]["vals"][:5] = 7.0
    bt.exec(1.0, 0.0)
    s.synchronize()
    old = _reference(dict(descs[-1], vals=v), 1.0, 0.0, np.zeros((m, 9)))[0]
    np.testing.assert_allclose(Cs[-1].cpu().numpy(), old, rtol=1e-5, atol=1e-5)
    bt.destroy()
    run_and_check()  # a new batch sees the new values
