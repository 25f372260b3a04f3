"""Benchmark of the sparse x dense execute path on B200.

Default workload (N=1): FP64 SELL-C-sigma SpMV on the power-law matrix
(n = 4,194,304 rows, row lengths Zipf-Mandelbrot p(k) ~ (k + q)^-2 on
[1, 4096] with q solved for mean 16, uniform unique columns, N(0,1) values,
x ~ U[-1,1], seed 1), C and sigma
picked by the exhaustive autotuner, compared with the plain CSR kernel on
the same matrix. A step is one y = A*x over the whole matrix with inputs
resident in HBM (889 MB of algorithmic traffic: larger than the 126 MB L2,
so no flush is needed between steps).

Reported:
  value      algorithmic GB/s of the tuned kernel (x, y and the matrix
             counted once, SELL padding not counted), summed over ranks;
  e2e        the same metric through the drop-in C call
             perflibs_spmv_exec_d with host (pinned) x and y: H2D of x and
             D2H of y inside every timed step (y comes back in row bands,
             each band's copy overlapping the next band's kernels);
  roofline   the dominant kernel's achieved GB/s vs the measured HBM peak;
  cpu_baseline  the reference library (compiled from its own sources,
             OpenMP on all host cores) on the same matrix, same metric.

--impl reference times only the reference CPU implementation.
Multi-GPU (torchrun): independent replicas, one per GPU (the path needs no
exchange), max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from perf_libs_sparse_b200 import workloads as W  # noqa: E402

FALLBACK_HBM_GBS = 6650.0


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def max_over_ranks(value: float, device="cpu") -> float:
    """The maximum of a per-rank float over the default process group (the
    value itself without one). Every rank must call it at the same point."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_gbs(bytes_per_step: float, seconds_per_step: float, world: int) -> float:
    """Whole-job GB/s of `world` independent replicas, each moving
    bytes_per_step, timed by the slowest rank's seconds per step."""
    return bytes_per_step / seconds_per_step / 1e9 * world


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for nm, v in zip(names, s[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def load_traffic(workload: str):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get(workload)
    return None


def make_c2():
    m, n, rp, c, v = W.zipf_rows(4_194_304, seed=1)
    x = W.uniform_vector(n, 1)
    return m, n, rp, c, v, x


# ------------------------------------------------------------------ CPU leg


def cpu_reference_spmv(m, n, rp, c, v, x, reps: int, budget_s: float = 20.0):
    """The reference library on all host cores: create, hint MANY, optimize
    (its auditioner), then repeated perflibs_spmv_exec_d. Returns (GB/s,
    seconds per exec, optimize seconds, threads, kind, sample)."""
    import oracle

    threads = os.cpu_count() or 1
    kind = "reference" if oracle.ref_available() else "port"
    bytes_ = W.algorithmic_bytes_spmv(m, n, int(rp[-1]), 8, 8, False)
    y = np.zeros(m)
    if kind == "reference":
        A = oracle.RefMatrix.csr(m, n, rp, c, v)
        A.hint(60, 300)
        A.hint(80, 420)
        t0 = time.perf_counter()
        A.optimize()
        t_opt = time.perf_counter() - t0
        A.spmv(x, y)
        times = []
        t_start = time.perf_counter()
        for _ in range(reps):
            t0 = time.perf_counter()
            A.spmv(x, y)
            times.append(time.perf_counter() - t0)
            if time.perf_counter() - t_start > budget_s:
                break
        fmt = A.format()
        A.destroy()
        sample = (f"full matrix, {len(times)} perflibs_spmv_exec_d calls after perflibs_spmv_optimize "
                  f"(audition chose format {fmt[0]}, C={fmt[1]}, sigma={fmt[2]}); OMP threads={threads}")
    else:
        t_opt = 0.0
        oracle.csr_spmv(rp, c, v, x, y=y)
        times = []
        t_start = time.perf_counter()
        for _ in range(reps):
            t0 = time.perf_counter()
            oracle.csr_spmv(rp, c, v, x, y=y)
            times.append(time.perf_counter() - t0)
            if time.perf_counter() - t_start > budget_s:
                break
        sample = f"full matrix, {len(times)} CSR SpMV calls of the oracle port; OMP threads={threads}"
    sec = statistics.median(times)
    return bytes_ / sec / 1e9, sec, t_opt, threads, kind, sample


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    m, n, rp, c, v, x = make_c2()
    reps = max(1, args.warmup + args.steps)
    gbs, sec, t_opt, threads, kind, sample = cpu_reference_spmv(m, n, rp, c, v, x, reps, budget_s=120.0)
    line = {
        "metric": "SpMV GB/s (algorithmic bytes), FP64, power-law matrix",
        "value": gbs, "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "C2 power-law SpMV n=4194304 nnz=%d" % int(rp[-1]), "optimize_s": t_opt},
        "impl": "reference",
        "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    emit(line, args)
    return 0


# ------------------------------------------------------------------ GPU leg


def run_b200(args):
    import torch

    import perf_libs_sparse_b200 as pls

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)

    m, n, rp, c, v, x = make_c2()
    nnz = int(rp[-1])
    bytes_step = W.algorithmic_bytes_spmv(m, n, nnz, 8, 8, False)

    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream

    # Plain CSR baseline (the default kernel, no tuning).
    A_plain = pls.SpMat.csr(m, n, rp, c, v)
    A_plain.set_stream(sp)
    A_plain.hint(pls.HINT_SPMV_INVOCATIONS, pls.INVOCATIONS_SINGLE)
    assert A_plain.optimize() == 0

    # Tuned: the exhaustive autotuner picks kernel family, C, sigma, TPR.
    A = pls.SpMat.csr(m, n, rp, c, v)
    A.set_stream(sp)
    A.hint(pls.HINT_SPMV_OPERATION, pls.OPERATION_NOTRANS)
    A.hint(pls.HINT_SPMV_INVOCATIONS, pls.INVOCATIONS_MANY)
    t0 = time.perf_counter()
    assert A.optimize() == 0
    t_opt = time.perf_counter() - t0
    cfg = A.config()

    xd = torch.tensor(x, device=dev)
    yd = torch.zeros(m, dtype=torch.float64, device=dev)

    def step(M):
        M.spmv_dev(xd.data_ptr(), yd.data_ptr(), 1.0, 0.0, sp)

    def timed(M, K, Wm, label="untimed"):
        with torch.cuda.stream(stream):
            for _ in range(Wm):
                step(M)
            torch.cuda.synchronize()
            if world > 1:
                torch.distributed.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.nvtx.range_push(label)
            e0.record(stream)
            for _ in range(K):
                step(M)
            e1.record(stream)
            torch.cuda.synchronize()
            torch.cuda.nvtx.range_pop()
            ms = e0.elapsed_time(e1)
        return max_over_ranks(ms, dev) / K

    K, Wm = args.steps, max(args.warmup, 3)
    # Keep the GPU busy ~0.5 s before each timed region, so that the clock
    # samples see the kernel under load and every arm (tuned, plain CSR, the
    # selector's) is timed in the same sustained power state.
    soak = max(1, int(args.soak_seconds / max(bytes_step / 6.0e12, 1e-6)))

    def measure(M, label="untimed"):
        timed(M, soak, 1)
        return timed(M, K, Wm, label)

    with ClockSampler(local) as clk:
        ms_tuned = measure(A, "timed")
    ms_plain = measure(A_plain)

    # Parity of the timed result (full size) against the oracle.
    import oracle

    step(A)
    torch.cuda.synchronize()
    y_gpu = yd.cpu().numpy()
    y_ref = oracle.csr_spmv(rp, c, v, x)
    scale = oracle.csr_absdot(rp, c, v, x)
    den = np.maximum(np.abs(y_ref), scale)
    den[den == 0] = 1

    def rel_err(y):
        return float((np.abs(y - y_ref) / den).max())

    max_rel = rel_err(y_gpu)
    # FP64 inf-norm check of the result: ||y - y_ref||_inf / (||A||_inf ||x||_inf),
    # with ||A||_inf from the library's own FP64 norm.
    a_inf = float(A.norm(pls.NORM_INF))
    x_inf = float(np.abs(x).max())

    def inf_check(y):
        return float(np.abs(y - y_ref).max() / max(a_inf * x_inf, 1e-300))

    # The learned selector (the trained parameters shipped with the package)
    # picks the layout; FP64, FP32 and BF16 value storage, each timed like
    # the tuned arm and checked against the FP64 oracle.
    from perf_libs_sparse_b200 import selector as selmod

    selector_arms = {}
    S = selmod.default_selector()
    if S is not None:
        for name, storage, tol in (("fp64", pls.STORAGE_NATIVE, 1e-12),
                                   ("fp32", pls.STORAGE_FP32, 1e-5),
                                   ("bf16", pls.STORAGE_BF16, 1e-2)):
            As = pls.SpMat.csr(m, n, rp, c, v)
            As.set_stream(sp)
            As.set_storage(storage)
            As.hint(pls.HINT_SPMV_INVOCATIONS, pls.INVOCATIONS_MANY)
            As.set_tuner(pls.TUNE_SELECTOR)
            S.attach(As)
            t0 = time.perf_counter()
            assert As.optimize() == 0
            t_sel = time.perf_counter() - t0
            ms_s = measure(As)
            step(As)
            torch.cuda.synchronize()
            ys = yd.cpu().numpy()
            cfg_s = As.config()
            selector_arms[name] = {
                "format": {0: "CSR", 1: "SELL-C-sigma", 2: "CSR-split"}[cfg_s["kind"]],
                "C": cfg_s["C"], "sigma": cfg_s["sigma"], "tpr": cfg_s["tpr"],
                "ms_per_step": ms_s, "speedup_vs_plain_csr_fp64": ms_plain / ms_s,
                "max_rel_err": rel_err(ys), "tolerance": tol, "inf_norm_check": inf_check(ys),
                "optimize_s": t_sel,
            }
            As.destroy()
        selector_arms["fp64"]["regret_vs_exhaustive"] = selector_arms["fp64"]["ms_per_step"] / ms_tuned - 1.0

    # End to end through the drop-in call with pinned host buffers.
    xh = torch.tensor(x).pin_memory()
    yh = torch.zeros(m, dtype=torch.float64).pin_memory()
    lib = pls.lib()
    import ctypes as C

    xp, yp = C.c_void_p(xh.data_ptr()), C.c_void_p(yh.data_ptr())
    for _ in range(2):
        lib.perflibs_spmv_exec_d(pls.OPERATION_NOTRANS, 1.0, A.h, xp, 0.0, yp)
    Ke = max(3, min(K, 30))
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(Ke):
        st = lib.perflibs_spmv_exec_d(pls.OPERATION_NOTRANS, 1.0, A.h, xp, 0.0, yp)
        assert st == 0
    e2e_s = max_over_ranks((time.perf_counter() - t0) / Ke, dev)
    e2e_bands = A.host_bands_used()

    hbm, peak_kind = peaks()
    achieved = replica_gbs(bytes_step, ms_tuned * 1e-3, 1)  # per GPU
    info = A.exec_info()
    kernels_per_step = info["kernels_per_spmv"]
    workload = f"C2 power-law SpMV n={m} nnz={nnz}"
    line = {
        "metric": "SpMV GB/s (algorithmic bytes) vs B200 HBM roofline, FP64, tuned vs plain CSR",
        "value": replica_gbs(bytes_step, ms_tuned * 1e-3, world),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": K,
        "warmup": Wm,
        "ms_per_step": ms_tuned,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {
            "workload": workload,
            "format": {0: "CSR", 1: "SELL-C-sigma", 2: "CSR-split"}[cfg["kind"]],
            "C": cfg["C"], "sigma": cfg["sigma"], "tpr": cfg["tpr"], "col_bytes": cfg["col_bytes"],
            "sell_items": info["n_items"], "sell_split_chunks": info["n_split"],
            "algorithmic_bytes_per_step": bytes_step,
            "l2": "inputs (889 MB) exceed the 126 MB L2; no flush between steps",
            "optimize_s": t_opt,
            "parallelism": f"replicas x{world}",
        },
        "plain_csr": {"value": replica_gbs(bytes_step, ms_plain * 1e-3, world), "ms_per_step": ms_plain},
        "speedup_vs_plain_csr": ms_plain / ms_tuned,
        "max_rel_err": max_rel,
        "inf_norm_check": inf_check(y_gpu),
        "gflops": 2.0 * nnz / (ms_tuned * 1e-3) / 1e9 * world,
        "selector": selector_arms or None,
        "e2e": {"value": replica_gbs(bytes_step, e2e_s, world), "unit": "GB/s",
                "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": m * 8, "ms_per_step": e2e_s * 1e3,
                "row_bands": e2e_bands},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_source": peak_kind,
                     "traffic": load_traffic("c2_spmv_fp64")},
        "gpu_launches": K * kernels_per_step,
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        os.environ.setdefault("OMP_PROC_BIND", "close")
        gbs, sec, t_opt_cpu, threads, kind, sample = cpu_reference_spmv(m, n, rp, c, v, x, reps=40)
        line["cpu_baseline"] = {"value": gbs, "unit": "GB/s", "cores": threads, "kind": kind,
                                "sample": sample, "optimize_s": t_opt_cpu, "ms_per_step": sec * 1e3}
    if rank == 0:
        emit(line, args)
    A.destroy()
    A_plain.destroy()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_extra(args):
    """Non-default workloads, one JSON line each (N = 1):
    c1  FP64 CSR SpMV, 5-point Laplacian 512^2 (21 MB: L2-resident, so a
        256 MB buffer is written between steps and only the SpMV is timed);
    c3  CSR SpMM on the 27-point 128^3 stencil, k = --k, value storage
        --storage (native = FP64 A, B, C; fp32 / bf16 = FP32 B, C and FP32 /
        BF16 A values, FP32 accumulation), max relative error vs the FP64
        oracle reported;
    c4  the 512-instance uneven batch (FP32) in one persistent launch per
        step (a CUDA graph), row tile picked by the batch autotuner."""
    import torch

    import oracle
    import perf_libs_sparse_b200 as pls

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    hbm, peak_kind = peaks()
    K, Wm = args.steps, max(args.warmup, 3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(step, flush=None):
        with torch.cuda.stream(stream):
            for _ in range(Wm):
                step()
            torch.cuda.synchronize()
            if flush is None:
                e0.record(stream)
                for _ in range(K):
                    step()
                e1.record(stream)
                torch.cuda.synchronize()
                return e0.elapsed_time(e1) / K
            tot = 0.0
            for _ in range(K):
                flush()
                e0.record(stream)
                step()
                e1.record(stream)
                torch.cuda.synchronize()
                tot += e0.elapsed_time(e1)
            return tot / K

    line = {"n_gpus": 1, "steps": K, "warmup": Wm, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "data": "synthetic", "unit": "GB/s"}
    if args.workload == "c3spmv":
        # FP64 SpMV (tuned) on C3's matrix: the structured counterpart of C2,
        # where x gathers are neighbours instead of uniformly random.
        m, n, rp, c, v = W.stencil_27pt(128, seed=2)
        x = W.uniform_vector(n, 2)
        A = pls.SpMat.csr(m, n, rp, c, v)
        A.set_stream(sp)
        A.hint(pls.HINT_SPMV_INVOCATIONS, pls.INVOCATIONS_MANY)
        assert A.optimize() == 0
        P = pls.SpMat.csr(m, n, rp, c, v)
        P.set_stream(sp)
        P.hint(pls.HINT_SPMV_INVOCATIONS, pls.INVOCATIONS_SINGLE)
        assert P.optimize() == 0
        xd = torch.tensor(x, device="cuda")
        yd = torch.zeros(m, dtype=torch.float64, device="cuda")
        ms_plain = timed(lambda: P.spmv_dev(xd.data_ptr(), yd.data_ptr(), 1.0, 0.0, sp))
        ms = timed(lambda: A.spmv_dev(xd.data_ptr(), yd.data_ptr(), 1.0, 0.0, sp))
        torch.cuda.synchronize()
        y = yd.cpu().numpy()
        y_ref = oracle.csr_spmv(rp, c, v, x)
        sc = oracle.csr_absdot(rp, c, v, x)
        err = float((np.abs(y - y_ref) / np.maximum(np.maximum(np.abs(y_ref), sc), 1e-300)).max())
        b = W.algorithmic_bytes_spmv(m, n, int(rp[-1]), 8, 8, False)
        cfg = A.config()
        line.update(metric="SpMV GB/s (algorithmic bytes), FP64, 27-point stencil 128^3, tuned vs plain CSR",
                    dtype="f64", value=b / ms / 1e6, ms_per_step=ms, max_rel_err=err,
                    plain_csr={"value": b / ms_plain / 1e6, "ms_per_step": ms_plain},
                    speedup_vs_plain_csr=ms_plain / ms,
                    config={"workload": "27-point stencil 128^3 n=2097152 nnz=55742968 (C3's matrix)",
                            "format": {0: "CSR", 1: "SELL-C-sigma", 2: "CSR-split"}[cfg["kind"]],
                            "C": cfg["C"], "sigma": cfg["sigma"], "tpr": cfg["tpr"],
                            "l2": "inputs (711 MB) exceed L2; no flush"})
    elif args.workload == "c1":
        m, n, rp, c, v = W.laplacian_2d(512)
        x = W.uniform_vector(n, 0)
        A = pls.SpMat.csr(m, n, rp, c, v)
        A.set_stream(sp)
        assert A.optimize() == 0
        xd = torch.tensor(x, device="cuda")
        yd = torch.zeros(m, dtype=torch.float64, device="cuda")
        flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
        ms = timed(lambda: A.spmv_dev(xd.data_ptr(), yd.data_ptr(), 1.0, 0.0, sp),
                   flush=lambda: flush_buf.fill_(1))
        torch.cuda.synchronize()
        y = yd.cpu().numpy()
        y_ref = oracle.csr_spmv(rp, c, v, x)
        sc = oracle.csr_absdot(rp, c, v, x)
        err = float((np.abs(y - y_ref) / np.maximum(np.maximum(np.abs(y_ref), sc), 1e-300)).max())
        b = W.algorithmic_bytes_spmv(m, n, int(rp[-1]), 8, 8, False)
        line.update(metric="SpMV GB/s (algorithmic bytes), FP64, 2D Laplacian 512^2", dtype="f64",
                    value=b / ms / 1e6, ms_per_step=ms, max_rel_err=err,
                    config={"workload": "C1 Laplacian 512x512 n=262144 nnz=1308672", **A.config(),
                            "l2": "256 MB written between steps, SpMV alone timed"})
    elif args.workload == "c3":
        m, n, rp, c, v = W.stencil_27pt(128, seed=2)
        k = args.k
        B = np.random.default_rng(2).uniform(-1, 1, (n, k))
        native = args.storage == "native"
        dt = np.float64 if native else np.float32
        tdt = torch.float64 if native else torch.float32
        A = pls.SpMat.csr(m, n, rp, c, v.astype(dt))
        A.set_storage({"native": pls.STORAGE_NATIVE, "fp32": pls.STORAGE_FP32, "bf16": pls.STORAGE_BF16}[args.storage])
        A.set_stream(sp)
        assert A.optimize() == 0
        Bd = torch.tensor(B, dtype=tdt, device="cuda")
        Cd = torch.zeros((m, k), dtype=tdt, device="cuda")
        ms = timed(lambda: A.spmm_dev(Bd.data_ptr(), k, k, Cd.data_ptr(), k, 1.0, 0.0, sp))
        torch.cuda.synchronize()
        got = Cd.cpu().numpy().astype(np.float64)
        rows = np.random.default_rng(7).choice(m, 20000, replace=False)
        rows.sort()
        # error on a row sample against the FP64 oracle (same seeds)
        sub_rp = np.concatenate([[0], np.cumsum(rp[rows + 1] - rp[rows])]).astype(np.int32)
        idx = np.concatenate([np.arange(rp[r], rp[r + 1]) for r in rows])
        ref = oracle.csr_spmm(sub_rp, c[idx], v[idx], B, k)
        scale = oracle.csr_spmm(sub_rp, c[idx], np.abs(v[idx]), np.abs(B), k)
        err = float((np.abs(got[rows] - ref) / np.maximum(np.maximum(np.abs(ref), scale), 1e-300)).max())
        # FP64 inf-norm check on the same rows: max row sum |C - C_ref| over
        # ||A||_inf ||B||_inf (||A||_inf from the library's FP64 norm).
        inf_chk = float(np.abs(got[rows] - ref).sum(axis=1).max()
                        / max(float(A.norm(pls.NORM_INF)) * float(np.abs(B).sum(axis=1).max()), 1e-300))
        sv = 8 if native else (4 if args.storage == "fp32" else 2)
        sb = 8 if native else 4
        b = W.algorithmic_bytes_spmm(m, n, int(rp[-1]), k, sv, sb, False)
        line.update(metric=f"SpMM GB/s (algorithmic bytes), 27-point 128^3, k={k}, storage {args.storage}",
                    dtype={"native": "f64", "fp32": "f32", "bf16": "bf16 values, f32 accumulate"}[args.storage],
                    value=b / ms / 1e6, ms_per_step=ms, max_rel_err=err, inf_norm_check=inf_chk,
                    gflops=2.0 * int(rp[-1]) * k / ms / 1e6,
                    config={"workload": "C3 27-point stencil 128^3 n=2097152 nnz=55742968", "k": k,
                            "storage": args.storage, "l2": "inputs exceed L2; no flush",
                            "spmm": A.spmm_info()})
    elif args.workload == "c4":
        inst = W.batched_instances(512, seed=3)
        mats, Bs, Cs = [], [], []
        for d in inst:
            if d["kind"] == "bsr":
                mats.append(pls.SpMat.bsr(d["layout"], d["m"], d["n"], d["bs"], d["row_ptr"], d["col"], d["vals"]))
            else:
                mats.append(pls.SpMat.csr(d["m"], d["n"], d["row_ptr"], d["col"], d["vals"]))
            Bs.append(torch.tensor(d["B"], device="cuda"))
            Cs.append(torch.zeros((d["m"], d["k"]), dtype=torch.float32, device="cuda"))
        ks = [d["k"] for d in inst]
        bt = pls.Batch(mats, ks, [b_.data_ptr() for b_ in Bs], ks, [c_.data_ptr() for c_ in Cs], ks, stream=sp)
        tile, _ = bt.tune()
        ms = timed(lambda: bt.exec(1.0, 0.0))
        b = sum(W.algorithmic_bytes_spmm(d["m"], d["n"], W.instance_nnz(d), d["k"], 4, 4, False) for d in inst)
        line.update(metric="Batched SpMM GB/s (algorithmic bytes), 512 uneven FP32 instances, one persistent launch",
                    dtype="f32", value=b / ms / 1e6, ms_per_step=ms,
                    config={"workload": "C4 512 instances n in [1024, 65536], k in [1, 64]", "tile_rows": tile,
                            **bt.info(), **bt.stage_info(), "rows_total": int(sum(d["m"] for d in inst))})
    line["roofline"] = {"bound": "hbm", "achieved": line["value"], "peak": hbm, "unit": "GB/s",
                        "frac": line["value"] / hbm, "peak_source": peak_kind}
    emit(line, args)
    return 0


def emit(line, args):
    """Print the result line; with --log, also append it to that JSON-lines
    file (one object per run, so a series of runs is one log)."""
    text = json.dumps(line)
    print(text)
    if args.log:
        with open(args.log, "a") as f:
            f.write(text + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c3spmv", "c4"],
                    help="c2 (default, the headline) or one of the other configurations")
    ap.add_argument("--k", type=int, default=32, help="right-hand sides for --workload c3")
    ap.add_argument("--storage", default="native", choices=["native", "fp32", "bf16"])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--log", default=None, help="append the result line to this JSON-lines file")
    ap.add_argument("--soak-seconds", type=float, default=0.5,
                    help="untimed load before the timed region, so the clock samples see the GPU busy")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "c2":
        return run_extra(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
