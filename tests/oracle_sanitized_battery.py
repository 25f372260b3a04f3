"""Every entry point of the oracle restatement on edge-case and random
inputs, for a run against its AddressSanitizer / UndefinedBehaviorSanitizer
build (tests/test_oracle_sanitized.py starts it with the sanitizer runtime
preloaded). Results are checked against numpy where that is a one-liner, so
the battery also fails on wrong answers, not only on sanitizer reports."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import oracle  # noqa: E402


def random_csr(m, n, max_len, rng, empty=0.2):
    lens = rng.integers(0, max_len + 1, m)
    lens[rng.random(m) < empty] = 0
    lens = np.minimum(lens, n)
    rp = np.zeros(m + 1, np.int32)
    rp[1:] = np.cumsum(lens)
    col = np.concatenate([np.sort(rng.choice(n, l, replace=False)) for l in lens]).astype(np.int32) \
        if rp[-1] else np.zeros(0, np.int32)
    vals = rng.standard_normal(int(rp[-1]))
    return rp, col, vals


def dense_of(rp, col, vals, m, n):
    A = np.zeros((m, n))
    for i in range(m):
        A[i, col[rp[i]:rp[i + 1]]] += vals[rp[i]:rp[i + 1]]
    return A


def main():
    rng = np.random.default_rng(0)
    shapes = [(0, 0, 0), (1, 1, 1), (1, 5, 5), (7, 3, 3), (31, 17, 9), (64, 64, 64), (200, 150, 40)]
    for m, n, ml in shapes:
        rp, col, vals = random_csr(m, n, ml, rng)
        A = dense_of(rp, col, vals, m, n)
        x = rng.uniform(-1, 1, n)
        y0 = rng.uniform(-1, 1, m)
        for mode in (0, 1):
            y = oracle.csr_spmv(rp, col, vals, x, y=y0, alpha=1.5, beta=-0.5, mode=mode)
            assert np.allclose(y, 1.5 * A @ x - 0.5 * y0)
        yf = oracle.csr_spmv(rp, col, vals.astype(np.float32), x.astype(np.float32))
        assert np.allclose(yf, A @ x, atol=1e-4)
        xt = rng.uniform(-1, 1, m)
        yt = oracle.csr_spmv_trans(rp, col, vals, n, xt, y=np.ones(n), alpha=2.0, beta=1.0)
        assert np.allclose(yt, 2.0 * A.T @ xt + 1.0)
        assert np.allclose(oracle.csr_absdot(rp, col, vals, x), np.abs(A) @ np.abs(x))
        for C in (2, 4, 8, 16, 32):
            for sigma in (0, C, 4 * C):
                s = oracle.scs_build(rp, col, vals, n, C, sigma)
                if m:
                    assert np.allclose(oracle.scs_spmv(s, x), A @ x)
                    oracle.scs_beta(s, len(vals))
        B = rng.uniform(-1, 1, (n, 5))
        C0 = rng.uniform(-1, 1, (m, 5))
        got = oracle.csr_spmm(rp, col, vals, B, 5, Cmat=C0, alpha=0.5, beta=2.0)
        assert np.allclose(got, 0.5 * A @ B + 2.0 * C0)
        assert np.isclose(oracle.csr_inf_norm(rp, vals), np.abs(A).sum(1).max() if m else 0.0)
        if m and n:
            r = np.repeat(np.arange(m), np.diff(rp)).astype(np.int32)
            rp2, c2, v2 = oracle.coo2csr(m, n, r[::-1].copy(), col[::-1].copy(), vals[::-1].copy())
            assert np.allclose(dense_of(rp2, c2, v2, m, n), A)
            At = A.T
            cp = np.zeros(n + 1, np.int32)
            nzr, nzc = np.nonzero(At)
            np.add.at(cp, nzr + 1, 1)
            cp = np.cumsum(cp).astype(np.int32)
            rp3, c3, v3 = oracle.csc2csr(m, n, nzc.astype(np.int32), cp, At[nzr, nzc])
            assert np.allclose(dense_of(rp3, c3, v3, m, n), A)
    for bs in (1, 2, 3, 4, 8):
        for layout in (90, 91):
            mb, nb = 5, 4
            m, n = mb * bs, nb * bs
            rp, col, vals = random_csr(m, n, n, rng, empty=0.3)
            A = dense_of(rp, col, vals, m, n)
            brp, bcol, bvals = oracle.csr2bsr(rp, col, vals, m, n, bs, layout)
            x = rng.uniform(-1, 1, n)
            assert np.allclose(oracle.bsr_spmv(brp, bcol, bvals, bs, layout, x), A @ x)
            rp4, c4, v4 = oracle.bsr2csr(brp, bcol, bvals, bs, layout)
            assert np.allclose(dense_of(rp4, c4, v4, m, n), A)
    print("oracle battery ok")


if __name__ == "__main__":
    main()
