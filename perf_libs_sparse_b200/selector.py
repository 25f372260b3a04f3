"""Learned selector: dataset, training and evaluation.

The selector maps the 24 device-computed structure statistics of a matrix to
one of the exhaustive tuner's candidates (CSR threads-per-row, CSR long-row
split, SELL-C-sigma C x sigma). This module:

1. generates the synthetic corpus on the GPU (seeded torch RNG, five
   families: 2D/3D stencils, banded, power-law rows, uniform random rows,
   BSR-structured blocks; n log-uniform in [1e4, 2e6], nonzeros per row
   log-uniform in [3, 200], total nonzeros capped at NNZ_CAP so one pass
   over the corpus fits a GPU session);
2. for every matrix computes the features (perflibs_b200_spmat_features)
   and runs the exhaustive tuner (perflibs_spmv_optimize, tuner
   EXHAUSTIVE) whose timing table is the label and the reference for
   regret; progress is
   appended to a checkpoint file so an interrupted run resumes;
3. trains the MLP with the library's CUDA kernels
   (perflibs_b200_selector_train) on the training split and reports, on the
   held-out split, regret t_selected / t_best - 1 against the exhaustive
   tuner, and the speed-up over the plain FP64 CSR kernel and over the
   reference-style rule (first SELL layout with padding efficiency >= 0.96,
   src/matvec.cpp:302-327) — the method without the network.

Usage: python -m perf_libs_sparse_b200.selector --n 3000 --out DIR
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import time

import numpy as np

from . import (SpMat, _check, _p, lib, HINT_SPMV_INVOCATIONS, INVOCATIONS_MANY, KIND_CSR,
               KIND_CSR_SPLIT, KIND_SELL, TUNE_EXHAUSTIVE, TUNE_SELECTOR)

NF = 24
NNZ_CAP = 24_000_000
# Parameters of the selector trained on the generated corpus (written by
# `main`, shipped with the package).
SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "selector_params.npy")
FAMILIES = ("stencil", "banded", "powerlaw", "uniform", "blocks")
SOFT_TAU = 0.05


# ------------------------------------------------------------- bindings

def _bind():
    L = lib()
    vp, i32, i64, f, u64 = C.c_void_p, C.c_int32, C.c_int64, C.c_float, C.c_uint64
    for name, args in {
        "perflibs_b200_spmat_features": [vp, vp],
        "perflibs_b200_tune_candidates": [i32, vp, vp],
        "perflibs_b200_selector_create": [vp, i32, u64],
        "perflibs_b200_selector_destroy": [vp],
        "perflibs_b200_spmat_set_spmm_selectors": [vp, vp],
        "perflibs_b200_selector_get_params": [vp, vp],
        "perflibs_b200_selector_set_params": [vp, vp],
        "perflibs_b200_selector_loss_grad": [vp, vp, vp, i32, vp, vp],
        "perflibs_b200_selector_train": [vp, vp, vp, i32, i32, i32, f, u64, vp],
        "perflibs_b200_selector_predict": [vp, vp, i32, vp, vp],
        "perflibs_b200_spmat_set_selector": [vp, vp],
        "perflibs_b200_spmat_create_csr_d_dev": [vp, i32, i32, vp, vp, vp, vp],
    }.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.perflibs_b200_selector_param_count.argtypes = [vp]
    L.perflibs_b200_selector_param_count.restype = i64
    return L


def candidates():
    L = _bind()
    cnt = C.c_int32()
    L.perflibs_b200_tune_candidates(0, None, C.byref(cnt))
    cfg = np.zeros((cnt.value, 4), np.int32)
    L.perflibs_b200_tune_candidates(cnt.value, _p(cfg), C.byref(cnt))
    return cfg


def features(A: SpMat) -> np.ndarray:
    L = _bind()
    f = np.zeros(NF, np.float32)
    _check(L.perflibs_b200_spmat_features(A.h, _p(f)), "features")
    return f


class Selector:
    def __init__(self, n_classes: int, seed: int = 0):
        self.L = _bind()
        self.K = n_classes
        self.h = C.c_void_p()
        _check(self.L.perflibs_b200_selector_create(C.byref(self.h), n_classes, seed), "selector_create")

    @property
    def n_params(self):
        return int(self.L.perflibs_b200_selector_param_count(self.h))

    @property
    def n_trainable(self):
        return self.n_params - 2 * NF

    def get_params(self):
        p = np.zeros(self.n_params, np.float32)
        _check(self.L.perflibs_b200_selector_get_params(self.h, _p(p)), "get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _check(self.L.perflibs_b200_selector_set_params(self.h, _p(p)), "set_params")

    def loss_grad(self, X, T):
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        loss = C.c_float()
        g = np.zeros(self.n_trainable, np.float32)
        _check(self.L.perflibs_b200_selector_loss_grad(self.h, _p(X), _p(T), len(X), C.byref(loss), _p(g)),
               "loss_grad")
        return loss.value, g

    def train(self, X, T, epochs=300, batch=128, lr=3e-3, seed=0):
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        loss = C.c_float()
        _check(self.L.perflibs_b200_selector_train(self.h, _p(X), _p(T), len(X), epochs, batch, lr, seed,
                                                   C.byref(loss)), "train")
        return loss.value

    def predict(self, X):
        X = np.ascontiguousarray(X, np.float32)
        probs = np.zeros((len(X), self.K), np.float32)
        cls = np.zeros(len(X), np.int32)
        _check(self.L.perflibs_b200_selector_predict(self.h, _p(X), len(X), _p(probs), _p(cls)), "predict")
        return probs, cls

    def attach(self, A: SpMat):
        _check(self.L.perflibs_b200_spmat_set_selector(A.h, self.h), "set_selector")

    def save(self, path):
        np.save(path, self.get_params())

    def load(self, path):
        self.set_params(np.load(path))

    def __del__(self):
        try:
            if self.h:
                self.L.perflibs_b200_selector_destroy(self.h)
        except Exception:
            pass


def soft_targets(times: np.ndarray, tau: float = SOFT_TAU) -> np.ndarray:
    """Target distribution over candidates from measured times: weight
    exp(-(t/t_best - 1)/tau), normalised."""
    r = times / times.min(axis=1, keepdims=True) - 1.0
    w = np.exp(-r / tau)
    return (w / w.sum(axis=1, keepdims=True)).astype(np.float32)


# ------------------------------------------------------------- generators


def generate(idx: int, seed: int = 4):
    """Matrix `idx` of the corpus, on the GPU: (family, m, n, row_ptr, col,
    vals) with torch CUDA tensors (int32 / float64, 0-based)."""
    import torch

    rng = np.random.default_rng([seed, idx])
    fam = FAMILIES[idx % len(FAMILIES)]
    n = int(round(math.exp(rng.uniform(math.log(1e4), math.log(2e6)))))
    r = math.exp(rng.uniform(math.log(3), math.log(200)))
    r = min(r, NNZ_CAP / n)
    g = torch.Generator(device="cuda")
    g.manual_seed(int(rng.integers(0, 2**62)))
    dev = "cuda"

    def finish(rows, cols, m_, n_):
        key = rows.to(torch.int64) * n_ + cols.to(torch.int64)
        key = torch.unique(key)  # sorted, duplicates removed
        rows = (key // n_)
        cols = (key % n_).to(torch.int32)
        counts = torch.bincount(rows, minlength=m_)
        row_ptr = torch.zeros(m_ + 1, dtype=torch.int32, device=dev)
        row_ptr[1:] = torch.cumsum(counts, 0).to(torch.int32)
        vals = torch.randn(cols.numel(), generator=g, device=dev, dtype=torch.float64)
        return fam, m_, n_, row_ptr, cols, vals

    if fam == "stencil":
        three_d = rng.random() < 0.5
        if three_d:
            s = max(4, int(round(n ** (1 / 3))))
            m_ = s ** 3
            pts = 7 if rng.random() < 0.5 else 27
            i = torch.arange(m_, device=dev)
            z, y, x = i // (s * s), (i // s) % s, i % s
            offs = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
                    if pts == 27 or abs(dz) + abs(dy) + abs(dx) <= 1]
            rows, cols = [], []
            for dz, dy, dx in offs:
                ok = (z + dz >= 0) & (z + dz < s) & (y + dy >= 0) & (y + dy < s) & (x + dx >= 0) & (x + dx < s)
                rows.append(i[ok])
                cols.append((i + dz * s * s + dy * s + dx)[ok])
        else:
            s = max(4, int(round(math.sqrt(n))))
            m_ = s * s
            pts = 5 if rng.random() < 0.5 else 9
            i = torch.arange(m_, device=dev)
            y, x = i // s, i % s
            offs = [(dy, dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if pts == 9 or abs(dy) + abs(dx) <= 1]
            rows, cols = [], []
            for dy, dx in offs:
                ok = (y + dy >= 0) & (y + dy < s) & (x + dx >= 0) & (x + dx < s)
                rows.append(i[ok])
                cols.append((i + dy * s + dx)[ok])
        return finish(torch.cat(rows), torch.cat(cols), m_, m_)
    if fam == "banded":
        hb = int(max(1, min(n - 1, round(r * rng.uniform(0.5, 4.0)))))
        per = max(1, int(round(r)))
        rows = torch.arange(n, device=dev).repeat_interleave(per)
        off = torch.randint(-hb, hb + 1, (rows.numel(),), generator=g, device=dev)
        cols = (rows + off).clamp(0, n - 1)
        diag = torch.arange(n, device=dev)
        return finish(torch.cat([rows, diag]), torch.cat([cols, diag]), n, n)
    if fam == "powerlaw":
        # Zipf-Mandelbrot lengths with mean r (shift solved numerically).
        k = np.arange(1, 4097, dtype=np.float64)
        lo, hi = 0.0, 5000.0
        for _ in range(60):
            q = 0.5 * (lo + hi)
            p = (k + q) ** -2.0
            mean = (p * k).sum() / p.sum()
            lo, hi = (q, hi) if mean < r else (lo, q)
        p = (k + q) ** -2.0
        cdf = torch.tensor(np.cumsum(p / p.sum()), device=dev)
        u = torch.rand(n, generator=g, device=dev, dtype=torch.float64)
        lens = (torch.searchsorted(cdf, u) + 1).clamp(max=min(4096, n))
        rows = torch.arange(n, device=dev).repeat_interleave(lens)
        cols = torch.randint(0, n, (rows.numel(),), generator=g, device=dev)
        return finish(rows, cols, n, n)
    if fam == "uniform":
        lo_, hi_ = max(1, int(r * 0.5)), max(2, int(r * 1.5))
        lens = torch.randint(lo_, hi_ + 1, (n,), generator=g, device=dev).clamp(max=n)
        rows = torch.arange(n, device=dev).repeat_interleave(lens)
        cols = torch.randint(0, n, (rows.numel(),), generator=g, device=dev)
        return finish(rows, cols, n, n)
    # blocks: dense bs x bs blocks, block columns near the diagonal
    bs = int(rng.choice([2, 4, 8]))
    nb = max(2, n // bs)
    m_ = nb * bs
    bpr = max(1, int(round(r / bs)))
    brow = torch.arange(nb, device=dev).repeat_interleave(bpr)
    spread = max(1, int(nb * rng.uniform(0.001, 0.05)))
    bcol = (brow + torch.randint(-spread, spread + 1, (brow.numel(),), generator=g, device=dev)).clamp(0, nb - 1)
    ii, jj = torch.meshgrid(torch.arange(bs, device=dev), torch.arange(bs, device=dev), indexing="ij")
    rows = (brow[:, None] * bs + ii.reshape(-1)[None, :]).reshape(-1)
    cols = (bcol[:, None] * bs + jj.reshape(-1)[None, :]).reshape(-1)
    return finish(rows, cols, m_, m_)


def create_from_device(m, n, row_ptr, col, vals) -> SpMat:
    L = _bind()
    h = C.c_void_p()
    _check(L.perflibs_b200_spmat_create_csr_d_dev(C.byref(h), m, n, C.c_void_p(row_ptr.data_ptr()),
                                                   C.c_void_p(col.data_ptr()), C.c_void_p(vals.data_ptr()),
                                                   None), "create_csr_d_dev")
    return SpMat(h, np.float64)


# ------------------------------------------------------------------ SpMM
# The SpMM selector's classes (kSpmmClass in the library), the forced path
# (perflibs_b200_spmat_set_spmm_path) that runs each, and the path code that
# spmm_info reports when it did run; k of each bucket (k <= 16, 17..64, > 64)
# in the corpus.
SPMM_CLASSES = ("row group", "shared entries", "staged", "diagonal form", "diagonal form, TMA")
SPMM_FORCE = (0, 2, 1, 3, 4)
SPMM_KS = (8, 32, 128)
SHIPPED_SPMM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "selector_spmm_params.npz")


def spmm_library_times(t: np.ndarray) -> np.ndarray:
    """The candidate times the library's measured choice compares: the
    staged kernel is not a candidate where the diagonal form applies
    (infinite times are kernels that do not apply)."""
    t = np.array(t, np.float64, copy=True)
    dia = np.isfinite(t[..., 3])
    t[..., 2] = np.where(dia, np.inf, t[..., 2])
    return t


def spmm_pick(probs: np.ndarray, times: np.ndarray) -> np.ndarray:
    """The kernel the library runs from a prediction: the most probable
    class that applies (finite time); the row-group kernel always does."""
    order = np.argsort(-probs, axis=1, kind="stable")
    out = np.zeros(len(probs), np.int64)
    for i in range(len(probs)):
        for c in order[i]:
            if np.isfinite(times[i, c]):
                out[i] = c
                break
    return out


def time_spmm_kernels(A: SpMat, k: int, reps: int = 3) -> list:
    """Milliseconds of one FP64 SpMM with k right-hand sides and each kernel
    forced (SPMM_FORCE), inf for kernels that do not apply (the forced path
    fell back to another); A.m and A.n are set by the caller."""
    import torch

    Bd = torch.randn((A.n, k), dtype=torch.float64, device="cuda")
    Cd = torch.empty((A.m, k), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    # The SpMMs and both events on one explicit stream, so that the events
    # bracket them: a null stream handle would send the SpMMs to the
    # handle's own stream, which the legacy default stream's events do not
    # order against.
    st = torch.cuda.Stream()
    sp = st.cuda_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    out = []
    for cls, path in enumerate(SPMM_FORCE):
        A.set_spmm_path(path)
        A.spmm_dev(Bd.data_ptr(), k, k, Cd.data_ptr(), k, 1.0, 0.0, sp)
        torch.cuda.synchronize()
        if A.spmm_info()["path"] != path:
            out.append(float("inf"))
            continue
        e0.record(st)
        for _ in range(reps):
            A.spmm_dev(Bd.data_ptr(), k, k, Cd.data_ptr(), k, 1.0, 0.0, sp)
        e1.record(st)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1) / reps)
    A.set_spmm_path(-1)
    del Bd, Cd
    return out


def build_spmm_corpus(n_mats: int, out_dir: str, seed: int = 4, log_every: int = 50,
                      budget_s: float = 1e9):
    """Features and forced-kernel SpMM times (k in SPMM_KS) for the corpus
    matrices [0, n_mats) (the SpMV corpus's generators and seed), resumable;
    stops after budget_s seconds."""
    import torch

    os.makedirs(out_dir, exist_ok=True)
    ck = os.path.join(out_dir, "spmm_corpus.jsonl")
    done = {}
    if os.path.exists(ck):
        with open(ck) as f:
            for line in f:
                d = json.loads(line)
                done[d["idx"]] = d
    t0 = time.time()
    with open(ck, "a") as f:
        for i in range(n_mats):
            if i in done:
                continue
            if time.time() - t0 > budget_s:
                break
            fam, m, n, rp, col, vals = generate(i, seed)
            A = create_from_device(m, n, rp, col, vals)
            A.m, A.n = m, n
            feat = features(A)
            d = {"idx": i, "family": fam, "m": m, "n": n, "nnz": int(rp[-1].item()),
                 "features": feat.tolist(), "ms": {str(k): time_spmm_kernels(A, k) for k in SPMM_KS}}
            f.write(json.dumps(d, allow_nan=True) + "\n")
            f.flush()
            done[i] = d
            A.destroy()
            del rp, col, vals
            torch.cuda.empty_cache()
            if log_every and (i + 1) % log_every == 0:
                print(f"spmm corpus {i + 1}/{n_mats} {time.time() - t0:.0f}s", flush=True)
    return [done[i] for i in sorted(done)]


def evaluate_spmm(corpus, n_train: int, out_dir: str, epochs=400, batch=64, lr=3e-3, seed=0):
    """Train one 5-class selector per k bucket on the first n_train matrices
    and report, on the rest, the regret t_selected / t_best - 1 against the
    library's measured choice (the fastest applicable kernel) and the
    first-call timing the prediction saves (the measured choice runs each
    applicable kernel three times)."""
    X = np.array([d["features"] for d in corpus], np.float32)
    rep = {"n_train": int(n_train), "n_heldout": int(len(corpus) - n_train), "classes": list(SPMM_CLASSES),
           "buckets": {}}
    params = {}
    for b, k in enumerate(SPMM_KS):
        T = spmm_library_times(np.array([d["ms"][str(k)] for d in corpus], np.float64))
        Tt = np.where(np.isfinite(T), T, np.nan)
        best = np.nanmin(Tt, axis=1)
        r = np.where(np.isfinite(T), T / best[:, None] - 1.0, np.inf)
        w = np.exp(-r / SOFT_TAU)
        targets = (w / w.sum(axis=1, keepdims=True)).astype(np.float32)
        sel = Selector(len(SPMM_CLASSES), seed=seed + b)
        t0 = time.time()
        loss = sel.train(X[:n_train], targets[:n_train], epochs=epochs, batch=batch, lr=lr, seed=seed)
        train_s = time.time() - t0
        params[f"b{b}"] = sel.get_params()
        probs, _ = sel.predict(X[n_train:])
        Th = T[n_train:]
        pick = spmm_pick(probs, Th)
        chosen = Th[np.arange(len(Th)), pick]
        regret = chosen / best[n_train:] - 1.0
        rows_only = Th[:, 0] / best[n_train:] - 1.0
        timing_cost = 3.0 * np.where(np.isfinite(Th), Th, 0.0).sum(axis=1)  # the measured choice's runs
        rep["buckets"][str(k)] = {
            "train_final_loss": float(loss), "train_seconds": train_s,
            "regret_mean": float(regret.mean()), "regret_median": float(np.median(regret)),
            "regret_p90": float(np.percentile(regret, 90)),
            "top1_accuracy": float((pick == np.nanargmin(np.where(np.isfinite(Th), Th, np.nan), axis=1)).mean()),
            "row_group_only_regret_mean": float(rows_only.mean()),
            "first_call_timing_ms_saved_mean": float(timing_cost.mean()),
            "first_call_timing_over_one_spmm_mean": float((timing_cost / chosen).mean()),
            "best_class_counts": {SPMM_CLASSES[c]: int(v) for c, v in
                                  zip(*np.unique(np.nanargmin(np.where(np.isfinite(Th), Th, np.nan), axis=1),
                                                 return_counts=True))},
        }
    np.savez(os.path.join(out_dir, "selector_spmm_params.npz"), **params)
    with open(os.path.join(out_dir, "spmm_report.json"), "w") as f:
        json.dump(rep, f, indent=1)
    return rep


def default_spmm_selectors():
    """The shipped SpMM selectors (k <= 16, 17..64, > 64), or None."""
    if not os.path.exists(SHIPPED_SPMM):
        return None
    z = np.load(SHIPPED_SPMM)
    out = []
    for b in range(3):
        S = Selector(len(SPMM_CLASSES))
        S.set_params(z[f"b{b}"])
        out.append(S)
    return out


def attach_spmm_selectors(A: SpMat, sels):
    """Attach three SpMM selectors (or None) to a handle."""
    L = _bind()
    arr = (C.c_void_p * 3)(*[(s.h.value if s is not None else None) for s in (sels or [None] * 3)])
    _check(L.perflibs_b200_spmat_set_spmm_selectors(A.h, arr), "set_spmm_selectors")


def default_selector():
    """The shipped trained selector, or None when the package has none."""
    if not os.path.exists(SHIPPED):
        return None
    S = Selector(len(candidates()))
    S.load(SHIPPED)
    return S


# ---------------------------------------------------------------- corpus


def reference_rule(cands: np.ndarray, betas: np.ndarray, default_idx: int) -> int:
    """The reference's acceptance rule restated on this candidate set: SELL
    chunk heights in preference order (largest first), sigma in {0, 256,
    4096} (about the reference's C*{0, 200, 2000}); the first layout with
    padding efficiency beta >= 0.96 is used, else CSR
    (src/matvec.cpp:302-327)."""
    for Cc in (32, 16, 8):
        for sg in (0, 256, 4096):
            for i, c in enumerate(cands):
                if c[0] == KIND_SELL and c[1] == Cc and c[2] == sg and betas[i] >= 0.96:
                    return i
    return default_idx


def build_corpus(n_mats: int, out_dir: str, seed: int = 4, log_every: int = 50):
    """Features + exhaustive timings for matrices [0, n_mats), resumable."""
    import torch

    os.makedirs(out_dir, exist_ok=True)
    ck = os.path.join(out_dir, "corpus.jsonl")
    done = {}
    if os.path.exists(ck):
        with open(ck) as f:
            for line in f:
                d = json.loads(line)
                done[d["idx"]] = d
    cands = candidates()
    t0 = time.time()
    with open(ck, "a") as f:
        for i in range(n_mats):
            if i in done:
                continue
            fam, m, n, rp, col, vals = generate(i, seed)
            A = create_from_device(m, n, rp, col, vals)
            feat = features(A)
            A.hint(HINT_SPMV_INVOCATIONS, INVOCATIONS_MANY)
            A.set_tuner(TUNE_EXHAUSTIVE)
            _check(A.optimize(), "optimize")
            cfg, ms, betas = A.tune_table(with_beta=True)
            assert len(ms) == len(cands)
            nnz = int(rp[-1].item())
            d = {"idx": i, "family": fam, "m": m, "n": n, "nnz": nnz, "features": feat.tolist(),
                 "ms": ms.tolist(), "beta": betas.tolist()}
            f.write(json.dumps(d) + "\n")
            f.flush()
            done[i] = d
            A.destroy()
            del rp, col, vals
            torch.cuda.empty_cache()
            if log_every and (i + 1) % log_every == 0:
                print(f"corpus {i + 1}/{n_mats} {time.time() - t0:.0f}s", flush=True)
    return [done[i] for i in range(n_mats)]


def evaluate(corpus, n_train: int, out_dir: str, epochs=400, batch=128, lr=3e-3, seed=0):
    cands = candidates()
    X = np.array([d["features"] for d in corpus], np.float32)
    Tm = np.array([d["ms"] for d in corpus], np.float64)
    nnz = np.array([d["nnz"] for d in corpus], np.float64)
    m = np.array([d["m"] for d in corpus], np.float64)
    n = np.array([d["n"] for d in corpus], np.float64)
    Ttr = soft_targets(Tm[:n_train])
    sel = Selector(len(cands), seed=seed)
    t0 = time.time()
    loss = sel.train(X[:n_train], Ttr, epochs=epochs, batch=batch, lr=lr, seed=seed)
    train_s = time.time() - t0
    sel.save(os.path.join(out_dir, "selector_params.npy"))
    _, cls = sel.predict(X[n_train:])
    Th = Tm[n_train:]
    best = Th.min(1)
    chosen = Th[np.arange(len(Th)), cls]
    regret = chosen / best - 1.0
    # plain FP64 CSR: the default kernel (threads per row = 2^floor(log2 mean))
    mean_len = nnz[n_train:] / np.maximum(m[n_train:], 1)
    tpr = np.clip(2 ** np.floor(np.log2(np.maximum(mean_len, 1))), 1, 32).astype(int)
    plain_idx = np.array([int(np.flatnonzero((cands[:, 0] == KIND_CSR) & (cands[:, 3] == t))[0]) for t in tpr])
    plain = Th[np.arange(len(Th)), plain_idx]
    betas = np.array([d["beta"] for d in corpus[n_train:]], np.float64)
    rule_idx = np.array([reference_rule(cands, betas[i], plain_idx[i]) for i in range(len(Th))])
    rule = Th[np.arange(len(Th)), rule_idx]
    bytes_ =nnz[n_train:] * 12 + (m[n_train:] + 1) * 4 + n[n_train:] * 8 + m[n_train:] * 8
    rep = {
        "n_train": int(n_train), "n_heldout": int(len(Th)), "n_classes": int(len(cands)),
        "train_final_loss": float(loss), "train_seconds": train_s,
        "regret_mean": float(regret.mean()), "regret_p90": float(np.percentile(regret, 90)),
        "regret_median": float(np.median(regret)),
        "top1_accuracy": float((cls == Th.argmin(1)).mean()),
        "speedup_vs_plain_csr_geomean": float(np.exp(np.log(plain / chosen).mean())),
        "exhaustive_speedup_vs_plain_csr_geomean": float(np.exp(np.log(plain / best).mean())),
        "speedup_vs_reference_rule_geomean": float(np.exp(np.log(rule / chosen).mean())),
        "reference_rule_regret_mean": float((rule / best - 1.0).mean()),
        "plain_csr_regret_mean": float((plain / best - 1.0).mean()),
        "heldout_gbs_selected_total": float(bytes_.sum() / (chosen.sum() * 1e-3) / 1e9),
        "heldout_gbs_plain_csr_total": float(bytes_.sum() / (plain.sum() * 1e-3) / 1e9),
    }
    with open(os.path.join(out_dir, "selector_report.json"), "w") as f:
        json.dump(rep, f, indent=1)
    return rep


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=3000)
    ap.add_argument("--train", type=int, default=None)
    ap.add_argument("--out", default="selector_out")
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=400)
    ap.add_argument("--spmm", action="store_true", help="the SpMM kernel selectors instead")
    ap.add_argument("--budget-s", type=float, default=1e9, help="stop building the corpus after this")
    args = ap.parse_args()
    if args.spmm:
        corpus = build_spmm_corpus(args.n, args.out, args.seed, budget_s=args.budget_s)
        if len(corpus) < args.n:
            print(f"spmm corpus stopped at the time budget: {len(corpus)} of {args.n}")
        n_train = args.train if args.train is not None else int(round(0.8 * len(corpus)))
        print(json.dumps(evaluate_spmm(corpus, n_train, args.out, epochs=args.epochs)))
        return
    corpus = build_corpus(args.n, args.out, args.seed)
    n_train = args.train if args.train is not None else int(round(0.8 * args.n))
    rep = evaluate(corpus, n_train, args.out, epochs=args.epochs)
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
