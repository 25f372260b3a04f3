"""Run one SpMV or SpMM case repeatedly (for profilers and quick timing).

    python -m perf_libs_sparse_b200.case --matrix zipf --rows 2097152 \
        --kind sell --C 16 --sigma 16384 --reps 10

Matrices: zipf (power-law rows, seed 1), lap2d (5-point Laplacian on a
sqrt(rows)^2 grid), st27 (27-point stencil on a cbrt(rows)^3 grid, seed 2).
--k > 0 runs SpMM with k right-hand sides instead of SpMV. --storage picks
the value storage (native, fp32, bf16). Prints one JSON line with the
per-call time measured with CUDA events.
"""
from __future__ import annotations

import argparse
import json
import math

import numpy as np

from . import (KIND_CSR, KIND_CSR_SPLIT, KIND_SELL, STORAGE_BF16, STORAGE_FP32, STORAGE_NATIVE, SpMat)
from . import workloads as W


def make(matrix: str, rows: int):
    if matrix == "zipf":
        return W.zipf_rows(rows, seed=1)
    if matrix == "lap2d":
        return W.laplacian_2d(int(round(math.sqrt(rows))))
    if matrix == "st27":
        return W.stencil_27pt(int(round(rows ** (1 / 3))), seed=2)
    raise ValueError(matrix)


def main():
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--matrix", default="zipf")
    ap.add_argument("--rows", type=int, default=1 << 21)
    ap.add_argument("--kind", default="sell", choices=["csr", "sell", "split", "tuned"])
    ap.add_argument("--C", type=int, default=32)
    ap.add_argument("--sigma", type=int, default=4096)
    ap.add_argument("--tpr", type=int, default=0)
    ap.add_argument("--k", type=int, default=0)
    ap.add_argument("--storage", default="native", choices=["native", "fp32", "bf16"])
    ap.add_argument("--fp32-api", action="store_true")
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--spmm-path", type=int, default=-1,
                    help="-1 measured choice, 0 row group, 1 staged, 2 row group with shared entries")
    args = ap.parse_args()

    m, n, rp, c, v = make(args.matrix, args.rows)
    dt = np.float32 if args.fp32_api else np.float64
    A = SpMat.csr(m, n, rp, c, v.astype(dt))
    A.set_storage({"native": STORAGE_NATIVE, "fp32": STORAGE_FP32, "bf16": STORAGE_BF16}[args.storage])
    if args.kind == "sell":
        A.force_config(KIND_SELL, args.C, args.sigma, 0)
    elif args.kind == "csr":
        A.force_config(KIND_CSR, 0, 0, args.tpr)
    elif args.kind == "split":
        A.force_config(KIND_CSR_SPLIT, 0, 0, args.tpr or 1024)
    assert A.optimize() == 0
    tdt = torch.float32 if args.fp32_api else torch.float64
    # A dedicated stream: the library's device entry points treat a NULL
    # stream as "the handle's own stream", so torch's default stream (handle
    # 0) would not be the stream the events below are recorded on.
    s = torch.cuda.Stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.k > 0:
        A.set_spmm_path(args.spmm_path)
        B = torch.rand((n, args.k), dtype=tdt, device="cuda") * 2 - 1
        Cm = torch.empty((m, args.k), dtype=tdt, device="cuda")
        run = lambda: A.spmm_dev(B.data_ptr(), args.k, args.k, Cm.data_ptr(), args.k, 1.0, 0.0, s.cuda_stream)
    else:
        x = torch.rand(n, dtype=tdt, device="cuda") * 2 - 1
        y = torch.empty(m, dtype=tdt, device="cuda")
        run = lambda: A.spmv_dev(x.data_ptr(), y.data_ptr(), 1.0, 0.0, s.cuda_stream)
    run()
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(args.reps):
        run()
    e1.record(s)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.reps
    nnz = int(rp[-1])
    sv = {"native": np.dtype(dt).itemsize, "fp32": 4, "bf16": 2}[args.storage]
    sx = np.dtype(dt).itemsize
    if args.k > 0:
        b = W.algorithmic_bytes_spmm(m, n, nnz, args.k, sv, sx, False)
    else:
        b = W.algorithmic_bytes_spmv(m, n, nnz, sv, sx, False)
    print(json.dumps({"matrix": args.matrix, "m": m, "nnz": nnz, "k": args.k, "config": A.config(),
                      "exec_info": A.exec_info(), "spmm": A.spmm_info() if args.k > 0 else None,
                      "ms": ms, "gbs": b / ms / 1e6, "bytes": b}))


if __name__ == "__main__":
    main()
