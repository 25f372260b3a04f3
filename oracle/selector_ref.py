"""CPU oracle for the selector — TEST INFRASTRUCTURE ONLY.

* ``features(row_ptr, col, n)``: the 24 structure statistics in the order of
  include/perflibs_b200.h, restated in numpy (FP64). Feature 23 is the
  reference's mgmd statistic (src/matrix_statistics.cpp:23-93: per row, the
  summed log of the gaps between consecutive columns divided by the row
  length, exponentiated, averaged over all rows).
* ``mlp_loss_grad(params, K, X, T)``: forward and backward of the MLP
  NF -> 64 -> 64 -> K with ReLU and softmax cross-entropy against soft
  targets, FP64, returning the mean loss and the gradient of the trainable
  parameters in the library's parameter order.
"""
from __future__ import annotations

import numpy as np

import oracle

NF = 24
H = 64


def _sell_size(row_ptr, C, sigma):
    s = oracle.port()
    sz = np.zeros(2, np.int64)
    m = len(row_ptr) - 1
    s.orc_scs_sizes(m, oracle._p(np.ascontiguousarray(row_ptr, np.int32)), C, sigma, oracle._p(sz))
    return int(sz[1])


def features(row_ptr, col, n):
    row_ptr = np.asarray(row_ptr, np.int64)
    col = np.asarray(col, np.int64)
    m = len(row_ptr) - 1
    nnz = int(row_ptr[-1] - row_ptr[0])
    L = np.diff(row_ptr).astype(np.float64)
    M, N = max(m, 1), max(n, 1)
    mean = L.sum() / M
    var = max(0.0, (L ** 2).sum() / M - mean ** 2)
    sd = np.sqrt(var)
    m3 = (L ** 3).sum() / M - 3 * mean * (L ** 2).sum() / M + 2 * mean ** 3
    m4 = ((L ** 4).sum() / M - 4 * mean * (L ** 3).sum() / M + 6 * mean ** 2 * (L ** 2).sum() / M
          - 3 * mean ** 4)
    skew = m3 / (var * sd) if var > 0 else 0.0
    kurt = m4 / (var * var) - 3.0 if var > 0 else 0.0

    def pct(q):
        # The device keeps exact bins below 4096 and power-of-two bins above.
        Li = np.diff(row_ptr)
        binned = np.where(Li < 4096, Li, 2.0 ** np.floor(np.log2(np.maximum(Li, 1))))
        s = np.sort(binned)
        k = int(np.ceil(q * m)) - 1
        return float(s[max(k, 0)]) if m else 0.0

    rows = np.repeat(np.arange(m), np.diff(row_ptr))
    d = np.abs(col - rows) if nnz else np.zeros(0)
    f = np.zeros(NF)
    f[0] = np.log2(m + 1.0)
    f[1] = np.log2(n + 1.0)
    f[2] = np.log2(nnz + 1.0)
    f[3] = mean
    f[4] = sd
    f[5] = skew
    f[6] = kurt
    f[7] = np.log2(1.0 + (L.min() if m else 0))
    f[8] = np.log2(1.0 + (L.max() if m else 0))
    f[9] = (L == 0).sum() / M
    f[10] = np.log2(1.0 + pct(0.50))
    f[11] = np.log2(1.0 + pct(0.90))
    f[12] = np.log2(1.0 + pct(0.99))
    f[13] = np.log2(max(1.0, L.max() / mean)) if mean > 0 else 0.0
    f[14] = d.sum() / nnz / N if nnz else 0.0
    f[15] = (d.max() if nnz else 0) / N
    f[16] = (d <= 32).sum() / nnz if nnz else 0.0
    for k, bs in zip((17, 18, 19), (2, 4, 8)):
        if nnz:
            nbc = -(-n // bs)
            keys = np.unique((rows // bs) * nbc + col // bs)
            f[k] = nnz / (bs * bs * len(keys))
    for k, (C, sg) in zip((20, 21, 22), ((8, 0), (32, 0), (32, 1024))):
        sz = _sell_size(row_ptr, C, sg) if nnz else 0
        f[k] = nnz / sz if sz else 1.0
    mg = 0.0
    for i in range(m):
        c = col[row_ptr[i]:row_ptr[i + 1]]
        if len(c):
            with np.errstate(divide="ignore"):
                lg = np.log(np.abs(np.diff(c).astype(np.float64))).sum() if len(c) > 1 else 0.0
            mg += np.exp(lg / len(c))
    f[23] = np.log2(1.0 + mg / M)
    return f


def split_params(p, K):
    o = 0

    def take(n):
        nonlocal o
        v = p[o:o + n]
        o += n
        return v

    W1 = take(H * NF).reshape(H, NF)
    b1 = take(H)
    W2 = take(H * H).reshape(H, H)
    b2 = take(H)
    W3 = take(K * H).reshape(K, H)
    b3 = take(K)
    mean = take(NF)
    istd = take(NF)
    return W1, b1, W2, b2, W3, b3, mean, istd


def mlp_loss_grad(params, K, X, T):
    p = np.asarray(params, np.float64)
    W1, b1, W2, b2, W3, b3, mean, istd = split_params(p, K)
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    B = X.shape[0]
    xn = (X - mean) * istd
    z1 = xn @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    z3 = h2 @ W3.T + b3
    z3 = z3 - z3.max(1, keepdims=True)
    lse = np.log(np.exp(z3).sum(1, keepdims=True))
    logp = z3 - lse
    loss = -(T * logp).sum() / B
    dz = (np.exp(logp) - T) / B
    gW3 = dz.T @ h2
    gb3 = dz.sum(0)
    dh2 = (dz @ W3) * (h2 > 0)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (h1 > 0)
    gW1 = dh1.T @ xn
    gb1 = dh1.sum(0)
    grad = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, grad


def mlp_predict(params, K, X):
    """Class scores (logits) of the MLP for feature rows X, FP64."""
    W1, b1, W2, b2, W3, b3, mean, istd = split_params(np.asarray(params, np.float64), K)
    xn = (np.asarray(X, np.float64) - mean) * istd
    h1 = np.maximum(xn @ W1.T + b1, 0)
    h2 = np.maximum(h1 @ W2.T + b2, 0)
    return h2 @ W3.T + b3
