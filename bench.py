"""Benchmark of the sparse x dense execute path on B200.

Default workload (N=1): FP64 SELL-C-sigma SpMV on the power-law matrix
(n = 4,194,304 rows, row lengths Zipf-Mandelbrot p(k) ~ (k + q)^-2 on
[1, 4096] with q solved for mean 16, uniform unique columns, N(0,1) values,
x ~ U[-1,1], seed 1), C and sigma (sigma in 32..8192) picked by the
exhaustive autotuner, compared with the plain CSR kernel on the same matrix.
A step is one y = A*x over the whole matrix with inputs resident in HBM
(889 MB of algorithmic traffic: larger than the 126 MB L2, so no flush is
needed between steps).

Reported on the one line:
  value      algorithmic GB/s of the tuned kernel (x, y and the matrix
             counted once, SELL padding not counted), summed over ranks;
  e2e        the same metric through the drop-in C call
             perflibs_spmv_exec_d with host (pinned) x and y: H2D of x and
             D2H of y inside every timed step (y comes back in row bands,
             each band's copy overlapping the next band's kernels);
  roofline   the dominant kernel's achieved GB/s vs the measured HBM peak;
  cpu_baseline  the reference library (compiled from its own sources,
             OpenMP on all host cores) on the same matrix, same metric;
  configs    the other matrix configurations, each with its own time,
             roofline and max relative error against the FP64 oracle:
             c1 (5-point Laplacian 512^2, plain FP64 CSR SpMV, timed over
             rotating copies so that L2 cannot hold them), c3 (CSR SpMM on
             the 27-point 128^3 stencil, k = 8 / 32 / 128 in FP64 and k = 32
             with FP32 / BF16 value storage) and c4 (512 uneven FP32 SpMMs
             in one persistent launch, a CUDA graph).

--impl reference times only the reference CPU implementation, on the same
metric, unit and workload as the default line.
Multi-GPU (torchrun): independent replicas, one per GPU (the path needs no
exchange), max time over ranks; the extra configurations run at N = 1 only.
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
# The headline metric, printed identically by both arms (this library on the
# GPU and the reference library on the host cores).
METRIC = "SpMV/SpMM GB/s vs B200 HBM roofline; tuned vs plain CSR at ≤1e-12 rel err"
C2_WORKLOAD = "C2 power-law SpMV n=4194304 nnz={nnz}, FP64, sigma in 32..8192"
SIGMA_RANGE = (32, 8192)
KIND_NAMES = {0: "CSR", 1: "SELL-C-sigma", 2: "CSR-split"}


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


def load_traffic(workload: str, kernel: str):
    """DRAM bytes (read + write) of one launch of the configuration's
    dominant kernel, from the ncu capture summarised in
    profiles/traffic.json, or None when that file holds no capture of this
    kernel and layout (`kernel` names both, as the file records them)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f).get(workload)
        if isinstance(d, dict) and d.get("kernel") == kernel:
            return d.get("bytes")
    return None


def make_c2():
    m, n, rp, c, v = W.zipf_rows(4_194_304, seed=1)
    x = W.uniform_vector(n, 1)
    return m, n, rp, c, v, x


def roofline(gbs: float, traffic=None):
    hbm, kind = peaks()
    return {"bound": "hbm", "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
            "peak_source": kind, "traffic": traffic}


# ------------------------------------------------------------------ parity
# The FP64 oracle (the reference algorithm restated in C, oracle/) checks each
# timed result after its timing.


def spmv_rel_err(y, rp, c, v, x):
    """max_i |y_i - y_ref_i| / max(|y_ref_i|, sum_j |a_ij x_j|)."""
    import oracle

    y_ref = oracle.csr_spmv(rp, c, v, x)
    den = np.maximum(np.abs(y_ref), oracle.csr_absdot(rp, c, v, x))
    den[den == 0] = 1
    return float((np.abs(y - y_ref) / den).max()), y_ref


def spmm_rel_err_rows(get_rows, rp, c, v, B, k, blocks):
    """Per-row scaled error of C = A*B over the row blocks [r0, r1): the
    reference is the FP64 oracle on A's FP64 values and the FP64 B; the
    scale of row i is sum_j |a_ij| |B_j|. get_rows(r0, r1) returns the
    computed rows as an FP64 array."""
    import oracle

    worst = 0.0
    for r0, r1 in blocks:
        p0, p1 = int(rp[r0]), int(rp[r1])
        sub = (rp[r0:r1 + 1] - rp[r0]).astype(np.int32)
        cc, vv = c[p0:p1], v[p0:p1]
        ref = oracle.csr_spmm(sub, cc, vv, B, k)
        scale = oracle.csr_spmm(sub, cc, np.abs(vv), np.abs(B), k)
        got = get_rows(r0, r1)
        den = np.maximum(np.abs(ref), scale)
        den[den == 0] = 1
        worst = max(worst, float((np.abs(got - ref) / den).max()))
    return worst


def row_blocks(m: int, full: bool, block=16384, count=8):
    """All rows in blocks, or `count` blocks of `block` rows spread evenly
    (the first and the last included)."""
    if full:
        return [(r, min(m, r + 262144)) for r in range(0, m, 262144)]
    starts = np.linspace(0, m - block, count).astype(np.int64)
    return [(int(s), int(s) + block) for s in starts]


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
        # spmat_format_t (src/util.hpp:256-275): 0 CSR, 2 SELL-C-sigma.
        fname = {0: "CSR", 2: "SELL-C-sigma"}.get(fmt[0], f"format {fmt[0]}")
        sample = (f"full matrix, {len(times)} perflibs_spmv_exec_d calls after perflibs_spmv_optimize "
                  f"(its audition chose {fname}, C={fmt[1]}, sigma={fmt[2]}); OMP threads={threads}")
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
        "metric": METRIC,
        "value": gbs, "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": C2_WORKLOAD.format(nnz=int(rp[-1])), "optimize_s": t_opt},
        "impl": "reference",
        "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    emit(line, args)
    return 0


# ------------------------------------------------------------------ GPU leg


class Timer:
    """CUDA-event timing on one stream: W untimed steps, then K steps under
    one event pair (a synchronize and, with a process group, a barrier on
    both sides)."""

    def __init__(self, stream, world=1, device=None):
        import torch

        self.torch = torch
        self.stream = stream
        self.world = world
        self.device = device

    def __call__(self, step, K, Wm, label=None):
        torch = self.torch
        with torch.cuda.stream(self.stream):
            for _ in range(Wm):
                step()
            torch.cuda.synchronize()
            if self.world > 1:
                torch.distributed.barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            if label:
                torch.cuda.nvtx.range_push(label)
            e0.record(self.stream)
            for _ in range(K):
                step()
            e1.record(self.stream)
            torch.cuda.synchronize()
            if label:
                torch.cuda.nvtx.range_pop()
            ms = e0.elapsed_time(e1)
        return max_over_ranks(ms, self.device) / K


def timed_label(args):
    """NVTX range around the timed steps of a configuration run alone
    (--workload), which the ncu commands select with --nvtx-include timed/;
    inside the default line only the C2 steps carry it."""
    return "timed" if args.workload != "c2" else None


def c1_config(args, timer, sp):
    """C1: plain FP64 CSR SpMV on the 5-point Laplacian 512^2 (21 MB). One
    step is one SpMV; steps go round R copies of the matrix, x and y
    (R * 21 MB > 2 x 126 MB of L2), so every step reads its inputs from HBM.
    The R-step rounds are captured in one CUDA graph and K steps are timed
    under one event pair. The line is the plain CSR kernel (no tuning, the
    configuration's definition); "tuned" is the same measurement after the
    exhaustive autotuner (tuned once: the other copies share the structure,
    so their optimize applies the cached result)."""
    import torch

    import perf_libs_sparse_b200 as pls

    m, n, rp, c, v = W.laplacian_2d(512)
    x = W.uniform_vector(n, 0)
    nnz = int(rp[-1])
    b = W.algorithmic_bytes_spmv(m, n, nnz, 8, 8, False)
    R = 12

    def measure(invocations):
        mats, xs, ys = [], [], []
        for _ in range(R):
            A = pls.SpMat.csr(m, n, rp, c, v)
            A.set_stream(sp)
            A.hint(pls.HINT_SPMV_INVOCATIONS, invocations)
            assert A.optimize() == 0
            mats.append(A)
            xs.append(torch.tensor(x, device="cuda"))
            ys.append(torch.zeros(m, dtype=torch.float64, device="cuda"))

        def round_():
            for i in range(R):
                mats[i].spmv_dev(xs[i].data_ptr(), ys[i].data_ptr(), 1.0, 0.0, sp)

        graph = None
        try:
            round_()
            torch.cuda.synchronize()
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(graph, stream=timer.stream, capture_error_mode="thread_local"):
                round_()
            torch.cuda.synchronize()
            step = graph.replay
        except Exception:
            graph = None
            step = round_
        rounds = max(8, args.steps)
        ms = timer(step, rounds, max(args.warmup, 3), timed_label(args)) / R
        err = max(spmv_rel_err(y.cpu().numpy(), rp, c, v, x)[0] for y in (ys[0], ys[-1]))
        cfg = mats[0].config()
        gbs = b / ms / 1e6
        kname = (f"CSR threads-per-row {cfg['tpr']}" if cfg["kind"] == pls.KIND_CSR
                 else f"{KIND_NAMES[cfg['kind']]} C={cfg['C']} sigma={cfg['sigma']}")
        out = {"kernel": kname,
               "value": gbs, "unit": "GB/s", "ms_per_step": ms, "steps": rounds * R,
               "gflops": 2.0 * nnz / ms / 1e6, "max_rel_err": err, "tolerance": 1e-12,
               "graph": graph is not None,
               "roofline": roofline(gbs, load_traffic("c1_spmv_fp64", kname))}
        del graph
        for A in mats:
            A.destroy()
        return out

    plain = measure(pls.INVOCATIONS_SINGLE)
    tuned = measure(pls.INVOCATIONS_MANY)
    out = {"workload": f"C1 5-point Laplacian 512x512 n={m} nnz={nnz}, plain FP64 CSR SpMV",
           **plain,
           "l2": f"{R} rotating copies of matrix, x and y ({R * b / 1e6:.0f} MB) "
                 f"in {'one CUDA graph per round' if plain['graph'] else 'direct launches'}",
           "algorithmic_bytes_per_step": b,
           "tuned": tuned, "tuned_over_plain": plain["ms_per_step"] / tuned["ms_per_step"]}
    return out


def c3_config(args, timer, sp, arms):
    """C3: CSR SpMM C = A*B on the 27-point 128^3 stencil (n = 2,097,152,
    nnz = 55,742,968), B n x k row-major U[-1,1] (seed 2). Each arm is one
    (k, storage) pair; the kernel is the library's measured choice. A step
    is one SpMM; inputs exceed L2 at every k, so no flush."""
    import torch

    import perf_libs_sparse_b200 as pls
    from perf_libs_sparse_b200 import selector as selmod

    m, n, rp, c, v = W.stencil_27pt(128, seed=2)
    nnz = int(rp[-1])
    out = {"workload": f"C3 27-point stencil 128^3 n={m} nnz={nnz}, CSR SpMM C = A*B",
           "arms": []}
    kmax = max(k for k, _ in arms)
    Bfull = np.random.default_rng(2).uniform(-1, 1, (n, kmax))
    for k, storage in arms:
        B = np.ascontiguousarray(Bfull[:, :k]) if k < kmax else Bfull
        native = storage == "native"
        dt = np.float64 if native else np.float32
        tdt = torch.float64 if native else torch.float32
        A = pls.SpMat.csr(m, n, rp, c, v.astype(dt))
        A.set_storage({"native": pls.STORAGE_NATIVE, "fp32": pls.STORAGE_FP32,
                       "bf16": pls.STORAGE_BF16}[storage])
        A.set_stream(sp)
        if getattr(args, "spmm_path", None) is not None:
            A.set_spmm_path(args.spmm_path)
        assert A.optimize() == 0
        Bd = torch.tensor(B, dtype=tdt, device="cuda")
        Cd = torch.zeros((m, k), dtype=tdt, device="cuda")
        t0 = time.perf_counter()
        A.spmm_dev(Bd.data_ptr(), k, k, Cd.data_ptr(), k, 1.0, 0.0, sp)  # measured choice
        torch.cuda.synchronize()
        t_choice = time.perf_counter() - t0
        K = max(args.steps, 10)
        ms = timer(lambda: A.spmm_dev(Bd.data_ptr(), k, k, Cd.data_ptr(), k, 1.0, 0.0, sp),
                   K, max(args.warmup, 3), timed_label(args))
        torch.cuda.synchronize()
        full = k <= 32
        err = spmm_rel_err_rows(lambda r0, r1: Cd[r0:r1].cpu().numpy().astype(np.float64),
                                rp, c, v, B, k, row_blocks(m, full))
        sv = 8 if native else (4 if storage == "fp32" else 2)
        sb = 8 if native else 4
        b = W.algorithmic_bytes_spmm(m, n, nnz, k, sv, sb, False)
        gbs = b / ms / 1e6
        info = A.spmm_info()
        # The learned SpMM kernel selector on the same call: its first SpMM
        # runs the predicted kernel without timing the candidates.
        sel = None
        sels = selmod.default_spmm_selectors()
        if sels is not None and getattr(args, "spmm_path", None) is None:
            As = pls.SpMat.csr(m, n, rp, c, v.astype(dt))
            As.set_storage({"native": pls.STORAGE_NATIVE, "fp32": pls.STORAGE_FP32,
                            "bf16": pls.STORAGE_BF16}[storage])
            As.set_stream(sp)
            selmod.attach_spmm_selectors(As, sels)
            assert As.optimize() == 0
            t0 = time.perf_counter()
            As.spmm_dev(Bd.data_ptr(), k, k, Cd.data_ptr(), k, 1.0, 0.0, sp)
            torch.cuda.synchronize()
            t_pred = time.perf_counter() - t0
            pth = As.spmm_info()["path"]
            sel = {"kernel": SPMM_PATHS.get(pth, str(pth)), "same_as_measured": pth == info["path"],
                   "first_call_s": t_pred}
            if pth != info["path"]:
                ms_p = timer(lambda: As.spmm_dev(Bd.data_ptr(), k, k, Cd.data_ptr(), k, 1.0, 0.0, sp),
                             K, max(args.warmup, 3))
                sel.update({"ms_per_step": ms_p, "regret_vs_measured": ms_p / ms - 1.0})
            else:
                sel["regret_vs_measured"] = 0.0
            As.destroy()
        out["arms"].append({
            "k": k, "storage": storage,
            "dtype": {"native": "f64", "fp32": "f32 values, B and C; f32 accumulate",
                      "bf16": "bf16 values, f32 B and C; f32 accumulate"}[storage],
            "value": gbs, "unit": "GB/s", "ms_per_step": ms, "steps": K,
            "gflops": 2.0 * nnz * k / ms / 1e6, "max_rel_err": err,
            "tolerance": {"native": 1e-12, "fp32": 1e-5, "bf16": 1e-2}[storage],
            "rows_checked": "all" if full else "8 blocks of 16384 rows",
            "kernel": SPMM_PATHS.get(info["path"], str(info["path"])),
            "first_call_s": t_choice, "selector": sel, "algorithmic_bytes_per_step": b,
            "roofline": roofline(gbs, load_traffic(f"c3_spmm_k{k}_{storage}",
                                                   SPMM_PATHS.get(info["path"], "")))})
        del Bd, Cd
        A.destroy()
    return out


SPMM_PATHS = {-1: "none", 0: "row group", 1: "staged", 2: "row group, shared entries",
              3: "diagonal form", 4: "diagonal form, TMA-staged B", 5: "BSR tensor core"}


def make_batch(inst, sp):
    """A batch over `inst` (dicts of workloads.batched_instances): the
    handles, B on the device, C zeroed, one stream. Returns (batch, handles,
    B tensors, C tensors)."""
    import torch

    import perf_libs_sparse_b200 as pls

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
    return bt, mats, Bs, Cs


def c4_kinds_config(args, timer, sp):
    """C4's 512 instances split by kind, each part batched alone and tuned:
    banded, random (also by k: <= 4, 5-16, > 16), BSR, then all 512. A part
    alone holds less than the full step's bytes, so more of it stays in L2;
    the parts show where the full step's time goes."""
    import torch

    inst = W.batched_instances(512, seed=3)
    rnd = [d for d in inst if d["kind"] == "csr" and "band" not in d]
    parts = [("banded", [d for d in inst if "band" in d]), ("random", rnd),
             ("random k <= 4", [d for d in rnd if d["k"] <= 4]),
             ("random 4 < k <= 16", [d for d in rnd if 4 < d["k"] <= 16]),
             ("random k > 16", [d for d in rnd if d["k"] > 16]),
             ("bsr", [d for d in inst if d["kind"] == "bsr"]), ("all", inst)]
    out = {"workload": "C4's 512 instances by kind, each part batched alone and tuned", "parts": []}
    for name, sel in parts:
        bt, mats, Bs, Cs = make_batch(sel, sp)
        tile, _ = bt.tune()
        ms = timer(lambda: bt.exec(1.0, 0.0), max(args.steps, 10), max(args.warmup, 3))
        torch.cuda.synchronize()
        b = sum(W.algorithmic_bytes_spmm(d["m"], d["n"], W.instance_nnz(d), d["k"], 4, 4, False) for d in sel)
        out["parts"].append({"part": name, "instances": len(sel), "ms_per_step": ms, "value": b / ms / 1e6,
                             "unit": "GB/s", "algorithmic_bytes_per_step": b,
                             "multiply_adds": int(sum(W.instance_nnz(d) * d["k"] for d in sel)),
                             "tile_rows": tile, **bt.stage_info()})
        bt.destroy()
        for A in mats:
            A.destroy()
        del Bs, Cs
    return out


def c4_config(args, timer, sp):
    """C4: 512 uneven FP32 SpMMs (banded, random uniform and BSR
    block-diagonal instances, n in [1024, 65536], k in [1, 64], seed 3) in
    one persistent launch, replayed as a CUDA graph; tile schedule from the
    batch autotuner. A step is one batch launch (2.9 GB, beyond L2)."""
    import torch

    import oracle

    inst = W.batched_instances(512, seed=3)
    bt, mats, Bs, Cs = make_batch(inst, sp)
    tile, _ = bt.tune()
    K = max(args.steps, 10)
    ms = timer(lambda: bt.exec(1.0, 0.0), K, max(args.warmup, 3), timed_label(args))
    torch.cuda.synchronize()
    worst = 0.0
    for d, Cd in zip(inst, Cs):
        if d["kind"] == "bsr":
            rp, cc, vv = oracle.bsr2csr(d["row_ptr"], d["col"], d["vals"].astype(np.float64), d["bs"], d["layout"])
        else:
            rp, cc, vv = d["row_ptr"], d["col"], d["vals"].astype(np.float64)
        B = d["B"].astype(np.float64)
        ref = oracle.csr_spmm(rp, cc, vv, B, d["k"])
        scale = oracle.csr_spmm(rp, cc, np.abs(vv), np.abs(B), d["k"])
        den = np.maximum(np.abs(ref), scale)
        den[den == 0] = 1
        worst = max(worst, float((np.abs(Cd.cpu().numpy().astype(np.float64) - ref) / den).max()))
    b = sum(W.algorithmic_bytes_spmm(d["m"], d["n"], W.instance_nnz(d), d["k"], 4, 4, False) for d in inst)
    gbs = b / ms / 1e6
    si = bt.stage_info()
    ktag = f"k_batch_spmm (BSR blocks, band values) tile={tile} staging={bool(si.get('staging'))}"
    out = {"workload": "C4 512 uneven FP32 instances (banded / random / BSR bs 4-8), n in [1024, 65536], "
                       "k in [1, 64], one persistent launch per step",
           "value": gbs, "unit": "GB/s", "ms_per_step": ms, "steps": K, "max_rel_err": worst,
           "tolerance": 1e-5, "rows_checked": "all instances, all rows",
           "tile_rows": tile, **bt.info(), **si,
           "rows_total": int(sum(d["m"] for d in inst)), "algorithmic_bytes_per_step": b,
           "roofline": roofline(gbs, load_traffic("c4_batch_fp32", ktag))}
    bt.destroy()
    for A in mats:
        A.destroy()
    return out


def bsr8_config(args, timer, sp):
    """BSR SpMM with 8 x 8 blocks and BF16 value storage (FP32 B and C, FP32
    accumulation), the tensor-core kernel (tcgen05.mma kind::tf32) against the
    FMA kernel: (1) a blocked random matrix, 32,768 block rows of 8 distinct
    random block columns each (n = 262,144, 16.8 M stored values), k = 128,
    seed 5; (2) the BSR instances of the C4 batch one by one. Errors against
    the FP64 oracle of the FP32 values; tolerance 1e-2 (BF16 storage)."""
    import torch

    import oracle
    import perf_libs_sparse_b200 as pls

    rng = np.random.default_rng(5)
    mb, per_row, k = 32768, 8, 128
    rp = np.arange(0, (mb + 1) * per_row, per_row, dtype=np.int32)
    col = np.concatenate([np.sort(rng.choice(mb, per_row, replace=False)) for _ in range(mb)]).astype(np.int32)
    vals = rng.uniform(-1, 1, len(col) * 64).astype(np.float32)
    n = mb * 8
    A = pls.SpMat.bsr(pls.ROW_MAJOR, n, n, 8, rp, col, vals)
    A.set_storage(pls.STORAGE_BF16)
    A.set_stream(sp)
    B = rng.uniform(-1, 1, (n, k)).astype(np.float32)
    Bd = torch.tensor(B, device="cuda")
    Cd = torch.zeros((n, k), dtype=torch.float32, device="cuda")
    nbytes = len(col) * 64 * 2 + len(col) * 4 + (mb + 1) * 4 + 2 * n * k * 4
    out = {"workload": f"BSR bs=8, {mb} block rows x {per_row} random blocks, n={n}, k={k}, BF16 values, "
                       "FP32 B and C", "algorithmic_bytes_per_step": nbytes, "arms": {}}
    crp, cc, cv = oracle.bsr2csr(rp, col, vals.astype(np.float64), 8, pls.ROW_MAJOR)
    rows = np.arange(0, 16384)
    for name, path in (("tensor_core", 5), ("fma", 0)):
        A.set_spmm_path(path)
        K = max(args.steps, 10)
        ms = timer(lambda: A.spmm_dev(Bd.data_ptr(), k, k, Cd.data_ptr(), k, 1.0, 0.0, sp), K,
                   max(args.warmup, 3), timed_label(args))
        torch.cuda.synchronize()
        ran = A.spmm_info()["path"]
        sub = (crp[:len(rows) + 1]).astype(np.int32)
        p1 = int(crp[len(rows)])
        ref = oracle.csr_spmm(sub, cc[:p1], cv[:p1], B.astype(np.float64), k)
        scale = oracle.csr_spmm(sub, cc[:p1], np.abs(cv[:p1]), np.abs(B.astype(np.float64)), k)
        got = Cd[:len(rows)].cpu().numpy().astype(np.float64)
        den = np.maximum(np.abs(ref), scale)
        den[den == 0] = 1
        out["arms"][name] = {"path": ran, "ms_per_step": ms, "value": nbytes / ms / 1e6, "unit": "GB/s",
                             "max_rel_err": float((np.abs(got - ref) / den).max()),
                             "rows_checked": len(rows), "roofline": roofline(nbytes / ms / 1e6)}
    A.destroy()
    del Bd, Cd
    # C4's BSR instances, one SpMM each, BF16 storage
    inst = [d for d in W.batched_instances(512, seed=3) if d["kind"] == "bsr"]
    tot = {5: 0.0, 0: 0.0}
    worst = 0.0
    for d in inst:
        Ai = pls.SpMat.bsr(d["layout"], d["m"], d["n"], d["bs"], d["row_ptr"], d["col"], d["vals"])
        Ai.set_storage(pls.STORAGE_BF16)
        Ai.set_stream(sp)
        Bi = torch.tensor(d["B"], device="cuda")
        Ci = torch.zeros((d["m"], d["k"]), dtype=torch.float32, device="cuda")
        for path in (5, 0):
            Ai.set_spmm_path(path)
            tot[path] += timer(lambda: Ai.spmm_dev(Bi.data_ptr(), d["k"], d["k"], Ci.data_ptr(), d["k"], 1.0, 0.0, sp),
                               5, 2)
        torch.cuda.synchronize()
        Ai.destroy()
    out["c4_bsr_instances"] = {"count": len(inst), "bs": sorted({d["bs"] for d in inst}),
                               "ms_total_tensor_core": tot[5], "ms_total_fma": tot[0],
                               "note": "one SpMM per instance (sum of per-instance times); the tensor-core "
                                       "kernel applies to the bs = 8 instances, bs = 4 ones run the FMA kernel"}
    return out


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
    timer = Timer(stream, world, dev)

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

    K, Wm = args.steps, max(args.warmup, 3)
    # Keep the GPU busy ~0.5 s before each timed region, so that the clock
    # samples see the kernel under load and every arm (tuned, plain CSR, the
    # selector's) is timed in the same sustained power state.
    soak = max(1, int(args.soak_seconds / max(bytes_step / 6.0e12, 1e-6)))

    def measure(M, label=None):
        timer(lambda: step(M), soak, 1)
        return timer(lambda: step(M), K, Wm, label)

    with ClockSampler(local) as clk:
        ms_tuned = measure(A, "timed")
    ms_plain = measure(A_plain)

    # Parity of the timed result (full size) against the oracle.
    step(A)
    torch.cuda.synchronize()
    y_gpu = yd.cpu().numpy()
    max_rel, y_ref = spmv_rel_err(y_gpu, rp, c, v, x)
    import oracle

    den = np.maximum(np.abs(y_ref), oracle.csr_absdot(rp, c, v, x))
    den[den == 0] = 1

    def rel_err(y):
        return float((np.abs(y - y_ref) / den).max())

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
                "format": KIND_NAMES[cfg_s["kind"]],
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
    e2e_err = rel_err(yh.numpy())

    achieved = replica_gbs(bytes_step, ms_tuned * 1e-3, 1)  # per GPU
    info = A.exec_info()
    kernels_per_step = info["kernels_per_spmv"]
    line = {
        "metric": METRIC,
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
            "workload": C2_WORKLOAD.format(nnz=nnz),
            "format": KIND_NAMES[cfg["kind"]],
            "C": cfg["C"], "sigma": cfg["sigma"], "tpr": cfg["tpr"], "col_bytes": cfg["col_bytes"],
            "sigma_in_range": cfg["kind"] != pls.KIND_SELL or SIGMA_RANGE[0] <= cfg["sigma"] <= SIGMA_RANGE[1],
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
                "row_bands": e2e_bands, "max_rel_err": e2e_err},
        "roofline": roofline(achieved, load_traffic(
            "c2_spmv_fp64", f"k_sell C={cfg['C']} sigma={cfg['sigma']}" if cfg["kind"] == 1 else "")),
        "gpu_launches": K * kernels_per_step,
        "clocks": clk.summary(),
    }
    A.destroy()
    A_plain.destroy()
    del xd, yd
    if rank == 0 and world == 1 and not args.no_configs:
        torch.cuda.empty_cache()
        line["configs"] = {
            "c1": c1_config(args, timer, sp),
            "c3": c3_config(args, timer, sp, [(8, "native"), (32, "native"), (128, "native"),
                                              (32, "fp32"), (32, "bf16")]),
            "c4": c4_config(args, timer, sp),
            "bsr8": bsr8_config(args, timer, sp),
        }
    if rank == 0 and world == 1 and not args.no_cpu:
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        os.environ.setdefault("OMP_PROC_BIND", "close")
        gbs, sec, t_opt_cpu, threads, kind, sample = cpu_reference_spmv(m, n, rp, c, v, x, reps=40)
        line["cpu_baseline"] = {"value": gbs, "unit": "GB/s", "cores": threads, "kind": kind,
                                "sample": sample, "optimize_s": t_opt_cpu, "ms_per_step": sec * 1e3}
    if rank == 0:
        emit(line, args)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def run_extra(args):
    """One configuration alone, as its own JSON line (N = 1): c1, c3 (k =
    --k, storage --storage), c4, c4kinds (C4's instance kinds batched
    apart), c3spmv (FP64 SpMV, tuned, on C3's
    matrix: the structured counterpart of C2), lap2d (FP64 SpMV, tuned, on
    the 5-point Laplacian 4096^2) or c2local (C2's row lengths
    with every column drawn from 8192, so that x's gathers hit L1: what the
    C2 kernel does without its L2 gathers). The default line carries
    c1 / c3 / c4 too; these lines are for profiling one kernel."""
    import torch

    import perf_libs_sparse_b200 as pls

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    timer = Timer(stream)
    if args.workload == "c1":
        sub = c1_config(args, timer, sp)
    elif args.workload == "bsr8":
        sub = bsr8_config(args, timer, sp)
    elif args.workload == "c3":
        sub = c3_config(args, timer, sp, [(args.k, args.storage)])["arms"][0]
    elif args.workload == "c4":
        sub = c4_config(args, timer, sp)
    elif args.workload == "c4kinds":
        sub = c4_kinds_config(args, timer, sp)
    else:
        if args.workload == "c2local":
            # C2's row lengths and uniform random columns, drawn from 8192
            # columns: x (64 KB) stays in L1, so the gathers do not reach L2.
            m, n, rp, c, v = W.zipf_rows(4_194_304, seed=1, ncols=8192)
            x = W.uniform_vector(n, 1)
            what = (f"C2's Zipf row lengths with columns from 8192 (x in L1) m={m} nnz={int(rp[-1])}, "
                    "FP64 SpMV: the C2 kernel without its L2 gathers")
        elif args.workload == "lap2d":
            # the C1 operator on a 4096 x 4096 grid: a structured SpMV large
            # enough (0.3 GB) to stream at HBM speed
            m, n, rp, c, v = W.laplacian_2d(4096)
            x = W.uniform_vector(n, 0)
            what = f"5-point Laplacian 4096^2 n={m} nnz={int(rp[-1])}, FP64 SpMV"
        else:
            m, n, rp, c, v = W.stencil_27pt(128, seed=2)
            x = W.uniform_vector(n, 2)
            what = "27-point stencil 128^3 n=2097152 nnz=55742968 (C3's matrix), FP64 SpMV"
        A = pls.SpMat.csr(m, n, rp, c, v)
        A.set_stream(sp)
        A.hint(pls.HINT_SPMV_INVOCATIONS, pls.INVOCATIONS_MANY)
        if args.sell_config:
            # a given SELL layout instead of the tuner's pick (to compare one
            # layout across matrices)
            C_, sigma = (int(t) for t in args.sell_config.split(","))
            assert A.force_config(pls.KIND_SELL, C_, sigma, 0) == 0
        assert A.optimize() == 0
        P = pls.SpMat.csr(m, n, rp, c, v)
        P.set_stream(sp)
        P.hint(pls.HINT_SPMV_INVOCATIONS, pls.INVOCATIONS_SINGLE)
        assert P.optimize() == 0
        xd = torch.tensor(x, device="cuda")
        yd = torch.zeros(m, dtype=torch.float64, device="cuda")
        K, Wm = args.steps, max(args.warmup, 3)
        ms_plain = timer(lambda: P.spmv_dev(xd.data_ptr(), yd.data_ptr(), 1.0, 0.0, sp), K, Wm)
        ms = timer(lambda: A.spmv_dev(xd.data_ptr(), yd.data_ptr(), 1.0, 0.0, sp), K, Wm, "timed")
        torch.cuda.synchronize()
        err, _ = spmv_rel_err(yd.cpu().numpy(), rp, c, v, x)
        b = W.algorithmic_bytes_spmv(m, n, int(rp[-1]), 8, 8, False)
        cfg = A.config()
        sub = {"workload": what,
               "value": b / ms / 1e6, "unit": "GB/s", "ms_per_step": ms, "max_rel_err": err,
               "plain_csr": {"value": b / ms_plain / 1e6, "ms_per_step": ms_plain},
               "speedup_vs_plain_csr": ms_plain / ms, "format": KIND_NAMES[cfg["kind"]],
               "C": cfg["C"], "sigma": cfg["sigma"], "tpr": cfg["tpr"],
               "roofline": roofline(b / ms / 1e6)}
    line = {"metric": f"{args.workload} GB/s (algorithmic bytes) vs B200 HBM roofline",
            "n_gpus": 1, "warmup": max(args.warmup, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic", **sub}
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
    ap.add_argument("--workload", default="c2",
                    choices=["c1", "c2", "c3", "c3spmv", "c2local", "lap2d", "c4", "c4kinds", "bsr8"],
                    help="c2 (default: the headline line, with c1 / c3 / c4 inside it) or one "
                         "configuration alone")
    ap.add_argument("--k", type=int, default=32, help="right-hand sides for --workload c3")
    ap.add_argument("--sell-config", default=None,
                    help="C,sigma: SELL layout for --workload c2local / c3spmv instead of the tuner's")
    ap.add_argument("--storage", default="native", choices=["native", "fp32", "bf16"])
    ap.add_argument("--spmm-path", type=int, default=None,
                    help="--workload c3: force one SpMM kernel (perflibs_b200_spmat_set_spmm_path)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--no-configs", action="store_true", help="skip the c1 / c3 / c4 configurations")
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
