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


def _banded(n, hb, rng):
    rows = np.arange(n)
    lo = np.maximum(rows - hb, 0)
    hi = np.minimum(rows + hb, n - 1)
    lens = hi - lo + 1
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    col = (np.repeat(lo, lens) + np.arange(rp[-1]) - np.repeat(rp[:-1], lens)).astype(np.int32)
    return rp, col, rng.uniform(-1, 1, int(rp[-1])).astype(np.float32)


def test_batch_staged_items_against_oracle_and_per_warp_items():
    """Banded and block-diagonal instances have blocks of rows that read a
    narrow window of B's rows; the batch computes those from a copy of the
    window in shared memory, at most 32 columns of C per item (k = 33, 64
    and 70 take two or three column slices; k = 1, 3 and 5 a padded
    float4). Leading dimensions that are not multiples of 4 keep C's stores
    scalar. A random instance has no narrow windows and stays on the
    per-warp items. Results with the staged items on and off both match the
    oracle within the FP32 bound, for beta = 0 and beta != 0."""
    import torch

    rng = np.random.default_rng(21)
    mats, descs = [], []
    for n, hb, k, pad in [(3000, 2, 1, 0), (2500, 17, 3, 0), (4100, 64, 5, 0), (3000, 30, 8, 0),
                          (2000, 64, 32, 0), (2200, 9, 33, 3), (1800, 40, 64, 0), (1500, 5, 70, 1),
                          (2600, 64, 16, 2)]:
        rp, c, v = _banded(n, hb, rng)
        mats.append(pls.SpMat.csr(n, n, rp, c, v))
        descs.append(dict(kind="csr", row_ptr=rp, col=c, vals=v, m=n, n=n, k=k, ldb=k + pad, ldc=k + pad))
    for bs, k in [(4, 6), (8, 16), (4, 40)]:
        nb = 700
        blocks = rng.uniform(-1, 1, (nb, bs * bs)).astype(np.float32)
        blocks[rng.random((nb, bs * bs)) >= 0.6] = 0.0
        rp = np.arange(nb + 1, dtype=np.int32)
        col = np.arange(nb, dtype=np.int32)
        mats.append(pls.SpMat.bsr(pls.ROW_MAJOR, nb * bs, nb * bs, bs, rp, col, blocks.reshape(-1)))
        descs.append(dict(kind="bsr", row_ptr=rp, col=col, vals=blocks.reshape(-1), bs=bs,
                          layout=pls.ROW_MAJOR, m=nb * bs, n=nb * bs, k=k, ldb=k, ldc=k))
    m = 5000
    rp, c, v = W.random_csr(m, m, 10, rng)
    v = v.astype(np.float32)
    mats.append(pls.SpMat.csr(m, m, rp, c, v))
    descs.append(dict(kind="csr", row_ptr=rp, col=c, vals=v, m=m, n=m, k=12, ldb=12, ldc=12))
    Bs, Cs, C0s = [], [], []
    for d in descs:
        d["B"] = rng.uniform(-1, 1, (d["n"], d["k"])).astype(np.float32)
        Bfull = np.zeros((d["n"], d["ldb"]), np.float32)
        Bfull[:, :d["k"]] = d["B"]
        Bs.append(torch.tensor(Bfull, device="cuda"))
        c0 = rng.uniform(-1, 1, (d["m"], d["ldc"])).astype(np.float32)
        C0s.append(c0)
        Cs.append(torch.tensor(c0, device="cuda"))
    s = torch.cuda.Stream()
    bt = pls.Batch(mats, [d["k"] for d in descs], [b.data_ptr() for b in Bs], [d["ldb"] for d in descs],
                   [cm.data_ptr() for cm in Cs], [d["ldc"] for d in descs], stream=s.cuda_stream)
    info = bt.stage_info()
    assert info["staged_items"] > 0 and info["staging"]

    def check(alpha, beta):
        for cm, c0 in zip(Cs, C0s):
            cm.copy_(torch.tensor(c0, device="cuda"))
        torch.cuda.synchronize()
        bt.exec(alpha, beta)
        s.synchronize()
        for d, cm, c0 in zip(descs, Cs, C0s):
            k = d["k"]
            ref, scale = _reference(d, alpha, beta, c0[:, :k].astype(np.float64))
            got = cm.cpu().numpy()
            den = np.maximum(np.abs(ref), scale)
            den[den == 0] = 1
            assert (np.abs(got[:, :k].astype(np.float64) - ref) / den).max() <= 1e-5, (d["kind"], d["m"], k)
            np.testing.assert_array_equal(got[:, k:], c0[:, k:])  # padding columns untouched

    for staging in (True, False):
        bt.set_staging(staging)
        assert bt.stage_info()["staging"] is staging
        for tile in (8, 128):
            bt.set_tile(tile)
            check(1.0, 0.0)
        check(1.5, -0.5)
    best, ms = bt.tune()
    assert best > 0 and ms > 0
    check(0.5, 2.0)
    bt.destroy()


def test_batch_scattered_rows_unaligned_k_against_oracle():
    """Scattered CSR instances whose k is not on 16-byte vectors (ldb or ldc
    not a multiple of 4) read B by element: k = 17-64 one row at a time with
    32 lanes over C's columns, k = 100 in two column passes, smaller k with
    several rows per warp; an instance with aligned rows shares the batch.
    Empty rows, ldb / ldc wider than k (padding columns untouched), items of
    8 and 128 rows and the tuner's choice, beta != 0, and B changed in place
    between two execs (the second sees it: B is read at exec, not copied)
    all match the oracle."""
    import torch

    rng = np.random.default_rng(33)
    mats, descs = [], []
    for m, n, per_row, k, ldb, ldc in [(3000, 2500, 12, 5, 5, 5), (2000, 4000, 20, 7, 9, 8),
                                       (1500, 1500, 6, 13, 13, 15), (2500, 3000, 18, 57, 57, 57),
                                       (1000, 1200, 9, 3, 3, 3), (1800, 1800, 14, 20, 20, 20),
                                       (1200, 900, 25, 33, 34, 33), (900, 1300, 30, 100, 101, 103),
                                       (2100, 700, 40, 19, 19, 21), (600, 600, 1, 29, 29, 29)]:
        rp, c, v = W.random_csr(m, n, per_row, rng, empty_frac=0.05)
        v = v.astype(np.float32)
        mats.append(pls.SpMat.csr(m, n, rp, c, v))
        descs.append(dict(kind="csr", row_ptr=rp, col=c, vals=v, m=m, n=n, k=k, ldb=ldb, ldc=ldc))
    Bs, Cs, C0s = [], [], []
    for d in descs:
        Bs.append(torch.tensor(rng.uniform(-1, 1, (d["n"], d["ldb"])).astype(np.float32), device="cuda"))
        c0 = rng.uniform(-1, 1, (d["m"], d["ldc"])).astype(np.float32)
        C0s.append(c0)
        Cs.append(torch.tensor(c0, device="cuda"))
    s = torch.cuda.Stream()
    bt = pls.Batch(mats, [d["k"] for d in descs], [b.data_ptr() for b in Bs], [d["ldb"] for d in descs],
                   [cm.data_ptr() for cm in Cs], [d["ldc"] for d in descs], stream=s.cuda_stream)
    assert bt.info()["launches"] == 1

    def check(alpha, beta, c_in):
        bt.exec(alpha, beta)
        s.synchronize()
        outs = []
        for d, b, cm, c0 in zip(descs, Bs, Cs, c_in):
            k = d["k"]
            ref, scale = _reference(dict(d, B=b.cpu().numpy()[:, :k]), alpha, beta, c0[:, :k].astype(np.float64))
            got = cm.cpu().numpy()
            den = np.maximum(np.abs(ref), scale)
            den[den == 0] = 1
            assert (np.abs(got[:, :k].astype(np.float64) - ref) / den).max() <= 1e-5, (d["m"], k)
            np.testing.assert_array_equal(got[:, k:], c0[:, k:])
            outs.append(got)
        return outs

    for tile in (8, 128, 0):
        if tile:
            bt.set_tile(tile)
        else:
            assert bt.tune()[0] > 0
        for cm, c0 in zip(Cs, C0s):
            cm.copy_(torch.tensor(c0, device="cuda"))
        torch.cuda.synchronize()
        c1 = check(1.25, -0.5, C0s)
        with torch.cuda.stream(s):
            for b in Bs:
                b.mul_(-2.0).add_(0.25)
        s.synchronize()
        check(0.75, 1.0, c1)
    bt.destroy()
