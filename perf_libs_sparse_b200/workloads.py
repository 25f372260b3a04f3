"""Seeded synthetic matrices and vectors for the sparse x dense execute path.

Every generator is deterministic in its seed (numpy PCG64) so the GPU path,
the CPU oracle and the reference library all see identical inputs.

* ``laplacian_2d(512)``: 5-point Laplacian on a 512 x 512 grid, natural
  row order, diagonal 4, off-diagonals -1 (n = 262,144, nnz = 1,308,672).
* ``zipf_rows(4_194_304, seed=1)``: row lengths from a Zipf law of exponent
  2 clipped to [1, 4096], shifted (Zipf-Mandelbrot, P(k) ~ (k + q)^-2) with
  q chosen so that the mean row length is 16 — plain Zipf(2) on [1, 4096]
  has mean 5.4, so the shift is what makes the stated nnz ~ 16 n hold;
  columns uniform without duplicates within a row (sorted), values N(0, 1).
* ``stencil_27pt(128, seed=2)``: 27-point stencil on a 128^3 grid,
  off-diagonals U[-1, 1], diagonal 1 + sum |off-diagonals| (n = 2,097,152,
  nnz = 55,742,968).
* ``random_csr``: small irregular matrices for parity tests (empty rows,
  index base 0 or 1).
"""
from __future__ import annotations

import numpy as np

ZIPF_S = 2.0
ZIPF_MAX = 4096
ZIPF_MEAN = 16.0


def _zipf_shift(mean: float = ZIPF_MEAN, s: float = ZIPF_S, kmax: int = ZIPF_MAX) -> float:
    k = np.arange(1, kmax + 1, dtype=np.float64)

    def m(q):
        p = (k + q) ** -s
        return float((p * k).sum() / p.sum())

    lo, hi = 0.0, 1000.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if m(mid) < mean:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def laplacian_2d(g: int = 512):
    """5-point Laplacian on a g x g grid (CSR, 0-based, sorted columns)."""
    n = g * g
    i = np.arange(n, dtype=np.int64)
    r, c = i // g, i % g
    offs = [(-g, r > 0), (-1, c > 0), (0, np.ones(n, bool)), (1, c < g - 1), (g, r < g - 1)]
    cols = np.stack([i + o for o, _ in offs], 1)
    mask = np.stack([mk for _, mk in offs], 1)
    vals = np.where(np.arange(5) == 2, 4.0, -1.0)[None, :].repeat(n, 0)
    counts = mask.sum(1)
    row_ptr = np.zeros(n + 1, np.int32)
    row_ptr[1:] = np.cumsum(counts)
    return n, n, row_ptr, cols[mask].astype(np.int32), vals[mask].astype(np.float64)


def zipf_lengths(n: int, rng: np.random.Generator) -> np.ndarray:
    q = _zipf_shift()
    k = np.arange(1, ZIPF_MAX + 1, dtype=np.float64)
    p = (k + q) ** -ZIPF_S
    cdf = np.cumsum(p / p.sum())
    cdf[-1] = 1.0
    u = rng.random(n)
    return (np.searchsorted(cdf, u, side="right") + 1).astype(np.int64).clip(1, ZIPF_MAX)


def zipf_rows(n: int = 4_194_304, seed: int = 1, ncols: int | None = None):
    """Power-law row lengths, uniform unique columns per row, N(0,1) values."""
    ncols = n if ncols is None else ncols
    rng = np.random.default_rng(seed)
    lens = zipf_lengths(n, rng)
    lens = np.minimum(lens, ncols)
    nnz = int(lens.sum())
    rows = np.repeat(np.arange(n, dtype=np.int64), lens)
    cols = rng.integers(0, ncols, size=nnz, dtype=np.int64)
    key = rows * ncols + cols
    key.sort(kind="stable")
    while True:
        dup = np.flatnonzero(np.diff(key) == 0) + 1
        if dup.size == 0:
            break
        r = key[dup] // ncols
        key[dup] = r * ncols + rng.integers(0, ncols, size=dup.size, dtype=np.int64)
        key.sort(kind="stable")
    cols = (key % ncols).astype(np.int32)
    row_ptr = np.zeros(n + 1, np.int32)
    row_ptr[1:] = np.cumsum(lens)
    vals = rng.standard_normal(nnz)
    return n, ncols, row_ptr, cols, vals


def stencil_27pt(g: int = 128, seed: int = 2):
    """27-point stencil on a g^3 grid; diagonally dominant diagonal."""
    rng = np.random.default_rng(seed)
    n = g * g * g
    i = np.arange(n, dtype=np.int64)
    z, y, x = i // (g * g), (i // g) % g, i % g
    offs = []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                offs.append((dz * g * g + dy * g + dx, dz, dy, dx))
    offs.sort()
    cols = np.empty((n, 27), np.int64)
    mask = np.empty((n, 27), bool)
    for t, (o, dz, dy, dx) in enumerate(offs):
        cols[:, t] = i + o
        mask[:, t] = ((z + dz >= 0) & (z + dz < g) & (y + dy >= 0) & (y + dy < g)
                      & (x + dx >= 0) & (x + dx < g))
    del z, y, x
    diag_t = [t for t, o in enumerate(offs) if o[0] == 0][0]
    vals = rng.uniform(-1.0, 1.0, size=(n, 27))
    vals[~mask] = 0.0
    off_abs = np.abs(vals).sum(1) - np.abs(vals[:, diag_t])
    vals[:, diag_t] = 1.0 + off_abs
    counts = mask.sum(1)
    row_ptr = np.zeros(n + 1, np.int32)
    row_ptr[1:] = np.cumsum(counts)
    return n, n, row_ptr, cols[mask].astype(np.int32), vals[mask]


def banded_csr(n: int, half_bandwidth: int, rng: np.random.Generator):
    """Square matrix with the full band |i - j| <= half_bandwidth, values
    U[-1, 1]: (m, n, row_ptr, col, vals), 0-based."""
    rows = np.arange(n)
    lo = np.maximum(rows - half_bandwidth, 0)
    hi = np.minimum(rows + half_bandwidth, n - 1)
    lens = hi - lo + 1
    row_ptr = np.zeros(n + 1, np.int32)
    row_ptr[1:] = np.cumsum(lens)
    col = (np.repeat(lo, lens) + np.arange(row_ptr[-1]) - np.repeat(row_ptr[:-1], lens)).astype(np.int32)
    vals = rng.uniform(-1, 1, int(row_ptr[-1]))
    return n, n, row_ptr, col, vals


def random_csr(m: int, n: int, max_len: int, rng: np.random.Generator, base: int = 0,
               empty_frac: float = 0.1, dtype=np.float64):
    """Small irregular CSR with some empty rows (for parity tests)."""
    max_len = min(max_len, n)
    lens = rng.integers(0, max_len + 1, m)
    lens[rng.random(m) < empty_frac] = 0
    row_ptr = np.zeros(m + 1, np.int32)
    row_ptr[1:] = np.cumsum(lens)
    cols = [np.sort(rng.choice(n, int(l), replace=False)) for l in lens]
    col = np.concatenate(cols).astype(np.int32) if row_ptr[-1] else np.zeros(0, np.int32)
    vals = rng.standard_normal(int(row_ptr[-1])).astype(dtype)
    return (row_ptr + base).astype(np.int32), (col + base).astype(np.int32), vals


def _sorted_unique(a: np.ndarray) -> np.ndarray:
    """np.unique(a) for integer keys (sorted distinct values), by a sort and
    an adjacent-difference mask: the same array, without numpy's hash-set
    path, which is two orders of magnitude slower on these sizes."""
    a = np.sort(a)
    if a.size == 0:
        return a
    keep = np.empty(a.size, bool)
    keep[0] = True
    np.not_equal(a[1:], a[:-1], out=keep[1:])
    return a[keep]


def batched_instances(count: int = 512, seed: int = 3, n_lo: int = 1024, n_hi: int = 65536,
                      k_max: int = 64):
    """The uneven batch: `count` independent FP32 instances, n log-uniform in
    [n_lo, n_hi], k log-uniform in [1, k_max], of three kinds in turn:
    banded (full band, half-bandwidth 2-64), random uniform (4-32 unique
    columns per row), and BSR block-diagonal (block size 4 or 8, each
    diagonal block filled with probability 0.3-0.9 per entry, zeros kept as
    explicit block entries). Values U[-1, 1]. Returns a list of dicts with
    'kind' ('csr' or 'bsr'), 'm', 'n', 'k', the arrays, and 'B' (n x k)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi)))))
        k = int(round(np.exp(rng.uniform(0.0, np.log(k_max)))))
        kind = ("banded", "uniform", "bsr")[i % 3]
        if kind == "banded":
            hb = int(rng.integers(2, 65))
            rows = np.arange(n)
            lo = np.maximum(rows - hb, 0)
            hi = np.minimum(rows + hb, n - 1)
            lens = hi - lo + 1
            row_ptr = np.zeros(n + 1, np.int32)
            row_ptr[1:] = np.cumsum(lens)
            col = (np.repeat(lo, lens) + np.arange(row_ptr[-1]) - np.repeat(row_ptr[:-1], lens)).astype(np.int32)
            vals = rng.uniform(-1, 1, row_ptr[-1]).astype(np.float32)
            d = dict(kind="csr", m=n, n=n, row_ptr=row_ptr, col=col, vals=vals, band=hb)
        elif kind == "uniform":
            lens = rng.integers(4, 33, n)
            row_ptr = np.zeros(n + 1, np.int32)
            row_ptr[1:] = np.cumsum(lens)
            rows = np.repeat(np.arange(n, dtype=np.int64), lens)
            key = _sorted_unique(rows * n + rng.integers(0, n, row_ptr[-1]))
            rows = key // n
            counts = np.bincount(rows, minlength=n)
            row_ptr[1:] = np.cumsum(counts)
            col = (key % n).astype(np.int32)
            vals = rng.uniform(-1, 1, len(col)).astype(np.float32)
            d = dict(kind="csr", m=n, n=n, row_ptr=row_ptr, col=col, vals=vals)
        else:
            bs = int(rng.choice([4, 8]))
            nb = max(1, n // bs)
            n = nb * bs
            fill = rng.uniform(0.3, 0.9)
            blocks = rng.uniform(-1, 1, (nb, bs * bs)).astype(np.float32)
            blocks[rng.random((nb, bs * bs)) >= fill] = 0.0
            d = dict(kind="bsr", m=n, n=n, bs=bs, layout=91, row_ptr=np.arange(nb + 1, dtype=np.int32),
                     col=np.arange(nb, dtype=np.int32), vals=blocks.reshape(-1), fill=fill)
        d["k"] = k
        d["B"] = rng.uniform(-1, 1, (d["n"], k)).astype(np.float32)
        out.append(d)
    return out


def instance_nnz(d) -> int:
    """Stored entries of an instance (BSR counts whole blocks)."""
    if d["kind"] == "bsr":
        return len(d["col"]) * d["bs"] * d["bs"]
    return int(d["row_ptr"][-1])


def uniform_vector(n: int, seed: int, dtype=np.float64) -> np.ndarray:
    return np.random.default_rng(seed).uniform(-1.0, 1.0, n).astype(dtype)


def algorithmic_bytes_spmv(m: int, n: int, nnz: int, s_v: int, s_x: int, beta_nonzero: bool) -> int:
    """nnz*(s_v + 4) + (m+1)*4 + n*s_x + m*s_y*(2 if beta != 0 else 1)."""
    return nnz * (s_v + 4) + (m + 1) * 4 + n * s_x + m * s_x * (2 if beta_nonzero else 1)


def algorithmic_bytes_spmm(m: int, n: int, nnz: int, k: int, s_v: int, s_b: int,
                           beta_nonzero: bool) -> int:
    """nnz*(s_v + 4) + (m+1)*4 + n*k*s_B + m*k*s_C*(2 if beta != 0 else 1)."""
    return nnz * (s_v + 4) + (m + 1) * 4 + n * k * s_b + m * k * s_b * (2 if beta_nonzero else 1)
