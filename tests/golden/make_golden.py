"""Generate the committed golden fixtures under tests/golden/.

Run in a container where the reference library has been compiled from its
own sources (``make -C oracle ref``):

    python tests/golden/make_golden.py

Outputs:
* ``reference_kats.json`` — known-answer tests transcribed from the
  reference's own test programs (values read from their source text; each
  entry names the file:line it comes from).
* ``ref_outputs.npz`` — outputs of the reference library itself on small
  seeded inputs: SELL-C-sigma layouts from its csr2scs + gen_data_vectors
  (including C = 32, which the reference builds but never executes), and
  FP64 CSR / SELL SpMV results from its exec kernels.
* ``ref_spmm.npz`` — C = alpha*A*B (+ beta*C0) from the reference's own
  perflibs_spmm_exec_d on small seeded CSR and BSR matrices, k in
  {4, 8, 32, 128}: k = 4 takes its repeated-SpMV route
  (src/matmul.cpp:26-28,42-89), larger k its row-wise blocked loop
  (src/compressed_sparse_rows.cpp:1699-1764), BSR its CSR view
  (src/matmul.cpp:616-631).

The tests never run this script; they read the fixtures.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from perf_libs_sparse_b200 import workloads as W  # noqa: E402

KATS = {
    "spmv_basic_d": {
        "source": "test/spmv_basic_d.c:13-22",
        "m": 5, "n": 5,
        "row_ptr": [0, 2, 4, 7, 9, 12],
        "col": [0, 2, 1, 3, 1, 2, 3, 2, 3, 2, 3, 4],
        "vals": [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12],
        "x": [1, 1, 1, 1, 1],
        "alpha": 1.0, "beta": 0.0,
        "y": [3.0, 7.0, 18.0, 17.0, 33.0],
        "tol": 1e-12,
    },
    "bsr_row_major": {
        "source": "test/bsr_kernel_paths.c:13-52",
        "layout": 91, "m": 4, "n": 4, "bs": 2,
        "row_ptr": [0, 2, 4], "col": [0, 1, 0, 1],
        "vals": [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16],
        "x": [1, 2, 3, 4],
        "y_notrans": [44.0, 64.0, 124.0, 144.0],
        "y_trans": [78.0, 88.0, 118.0, 128.0],
        "tol": 1e-12,
    },
    "bsr_col_major": {
        "source": "test/bsr_kernel_paths.c:87-135",
        "layout": 90, "m": 4, "n": 4, "bs": 2,
        "row_ptr": [0, 1, 3], "col": [0, 0, 1],
        "vals": [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12],
        "inf_norm": 36.0,
        # The reference transposes the handle and scales it by 0.5, then
        # multiplies by x = 1: the same as 0.5 * A^T * x.
        "x": [1, 1, 1, 1],
        "alpha_trans": 0.5,
        "y_trans_scaled": [7.0, 11.0, 9.5, 11.5],
        "tol": 1e-12,
    },
    "matmul_variants_d": {
        "source": "test/matmul_variants_d.c:59-130",
        "row_ptr": [0, 2, 4, 6, 8], "col": [0, 2, 0, 1, 1, 2, 2, 3],
        "vals": [1.0, -1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0],
        "denseA": [1.0, 0.0, -1.0, 0.0, 2.0, 3.0, 0.0, 0.0, 0.0, 4.0, 5.0, 0.0, 0.0, 0.0, 6.0, 7.0],
        "denseB": [float(v) for v in range(1, 17)],
        "c_init": [1.0, -1.0, 0.5, 2.0, 0.0, 0.25, -0.5, 0.5, 1.0, 1.5, -1.5, 2.5, 3.0, -2.0, 4.0, 5.0],
        "alpha_notrans": 1.0, "alpha_trans": 1.5, "alpha_beta": 0.7, "beta": 1.0,
        "tol": 1e-12,
    },
    "matrix_kernel_ops_spmm": {
        "source": "test/matrix_kernel_ops.c:72-97",
        "row_ptr": [0, 2, 3, 5, 7], "col": [0, 2, 1, 2, 3, 0, 3],
        "vals": [1.0, 2.0, 3.0, 4.0, 1.0, 2.0, 5.0],
        "denseB": [1.0, 2.0, 0.0, 1.0, 3.0, 4.0, 0.0, 2.0, 5.0, 6.0, 1.0, 0.0, 7.0, 8.0, 0.0, 3.0],
        "tol": 1e-12,
    },
    "strategy_paths_d": {
        "source": "test/strategy_paths_d.c:21-114",
        "m": 4096, "width": 12, "n": 65536, "updated_row": 1234,
        "y_plain": 12.0, "y_updated_row": 13.0, "alpha": 2.0, "beta": 1.0, "y0": 3.0,
        "col_first": 0, "col_last_from_end": 5,
        "tol": 1e-7,
    },
    "csr_spmv_omp_paths_float": {
        "source": "test/csr_spmv_omp_paths.c:13-125",
        "m": 1536, "n": 12288, "alpha": 1.75, "beta": -0.5,
        "row_lengths_cycle": [7, 113, 19, 181, 5, 149, 37, 223],
        "start_rule": "(29*i + 17) % (n - len)",
        "tol": 2e-4,
    },
}


def small_cases():
    """Seeded small matrices: (name, m, n, row_ptr, col, vals, x, y0)."""
    rng = np.random.default_rng(1234)
    out = []
    shapes = [(1, 1, 1), (7, 5, 3), (33, 40, 9), (100, 150, 30), (257, 300, 60), (64, 64, 64),
              (300, 3000, 80), (1000, 2000, 12)]
    for idx, (m, n, ml) in enumerate(shapes):
        base = idx % 2
        rp, c, v = W.random_csr(m, n, ml, rng, base=base, empty_frac=0.15)
        x = rng.uniform(-1, 1, n)
        y0 = rng.uniform(-1, 1, m)
        out.append((f"case{idx}", m, n, rp, c, v, x, y0))
    # Power-law rows (a small version of the C2 generator).
    m, n, rp, c, v = W.zipf_rows(600, seed=7)
    out.append(("zipf600", m, n, rp, c, v, rng.uniform(-1, 1, n), rng.uniform(-1, 1, m)))
    # Laplacian 32x32.
    m, n, rp, c, v = W.laplacian_2d(32)
    out.append(("lap32", m, n, rp, c, v, rng.uniform(-1, 1, n), rng.uniform(-1, 1, m)))
    return out


def spmm_cases():
    """Seeded small SpMM inputs: (name, kind, dict of arrays, ks)."""
    rng = np.random.default_rng(4321)
    out = []
    m, n, rp, c, v = W.stencil_27pt(5, seed=5)
    out.append(("st27_5", "csr", dict(m=m, n=n, row_ptr=rp, col=c, vals=v, base=0), (4, 8, 32, 128)))
    rp, c, v = W.random_csr(160, 220, 24, rng, empty_frac=0.15)
    out.append(("rand160", "csr", dict(m=160, n=220, row_ptr=rp, col=c, vals=v, base=0), (4, 8, 32, 128)))
    rp, c, v = W.random_csr(90, 70, 12, rng, base=1, empty_frac=0.2)
    out.append(("rand90_b1", "csr", dict(m=90, n=70, row_ptr=rp, col=c, vals=v, base=1), (4, 8)))
    for bs, mb, nb in ((4, 12, 15), (8, 7, 9)):
        for layout in (90, 91):
            rpb = np.zeros(mb + 1, np.int32)
            cols = []
            for i in range(mb):
                cc = np.sort(rng.choice(nb, int(rng.integers(0, 5)), replace=False))
                cols.append(cc)
                rpb[i + 1] = rpb[i] + len(cc)
            colb = np.concatenate(cols).astype(np.int32)
            vb = rng.uniform(-1, 1, len(colb) * bs * bs)
            vb[rng.random(len(vb)) < 0.25] = 0.0  # explicit zeros inside blocks
            name = f"bsr{bs}_{'col' if layout == 90 else 'row'}"
            out.append((name, "bsr", dict(m=mb * bs, n=nb * bs, bs=bs, layout=layout, row_ptr=rpb,
                                          col=colb, vals=vb), (4, 8, 32)))
    return out


def spmm_fixtures():
    """Reference SpMM outputs: per case and k, alpha = 1.5 with a null C, and
    (k in {4, 32}) alpha = 0.75, beta = -0.5 with a dense C0."""
    rng = np.random.default_rng(8765)
    arrays = {}
    for name, kind, d, ks in spmm_cases():
        m, n = d["m"], d["n"]
        kmax = max(ks)
        B = rng.uniform(-1, 1, (n, kmax))
        C0 = rng.uniform(-1, 1, (m, kmax))
        for key, val in d.items():
            arrays[f"{name}/{key}"] = np.asarray(val)
        arrays[f"{name}/kind"] = np.array(0 if kind == "csr" else 1)
        arrays[f"{name}/B"] = B
        arrays[f"{name}/C0"] = C0
        arrays[f"{name}/ks"] = np.array(ks, np.int32)
        if kind == "csr":
            A = oracle.RefMatrix.csr(m, n, d["row_ptr"], d["col"], d["vals"])
        else:
            A = oracle.RefMatrix.bsr(d["layout"], m, n, d["bs"], d["row_ptr"], d["col"], d["vals"])
        for k in ks:
            Bk = np.ascontiguousarray(B[:, :k])
            arrays[f"{name}/C_k{k}"] = A.spmm(m, Bk, alpha=1.5)
            if k in (4, 32):
                C0k = np.ascontiguousarray(C0[:, :k])
                arrays[f"{name}/Cb_k{k}"] = A.spmm(m, Bk, alpha=0.75, beta=-0.5, C0=C0k)
        A.destroy()
    np.savez_compressed(os.path.join(HERE, "ref_spmm.npz"), **arrays)
    return len(arrays)


def main():
    assert oracle.ref_available(), "build the reference oracle first: make -C oracle ref"
    print("wrote", spmm_fixtures(), "SpMM arrays")
    with open(os.path.join(HERE, "reference_kats.json"), "w") as f:
        json.dump(KATS, f, indent=1)
    arrays = {}
    for name, m, n, rp, c, v, x, y0 in small_cases():
        arrays[f"{name}/row_ptr"] = rp
        arrays[f"{name}/col"] = c
        arrays[f"{name}/vals"] = v
        arrays[f"{name}/x"] = x
        arrays[f"{name}/y0"] = y0
        arrays[f"{name}/shape"] = np.array([m, n], np.int64)
        # Reference CSR exec, INVOCATIONS_SINGLE (no audition): the default
        # serial kernel, alpha=1.5, beta=-0.5.
        A = oracle.RefMatrix.csr(m, n, rp, c, v)
        A.hint(80, 400)
        A.optimize()
        y = y0.copy()
        assert A.spmv(x, y, alpha=1.5, beta=-0.5) == 0
        arrays[f"{name}/y_csr"] = y
        A.destroy()
        variants = ((4, 1), (8, 0), (8, 8), (16, 1), (32, 0), (32, 1), (32, 8))
        if len(c) > 8000:  # keep the fixture small: one layout for the big cases
            variants = ((32, 8),)
        for C, sm in variants:
            s = oracle.ref_scs_build(rp, c, v, n, C, C * sm)
            key = f"{name}/scs_C{C}_s{C * sm}"
            for fld in ("cs", "cl", "col_min", "permd2in", "vals"):
                arrays[f"{key}/{fld}"] = s[fld]
            arrays[f"{key}/offsets"] = s["offsets"].astype(np.int32)
            arrays[f"{key}/info"] = np.array(
                [s["nC"], s["C"], s["sigma"], s["col_bytes"], s["n_full_chunks"],
                 s["ntidyup"], s["size"]], np.int64)
    np.savez_compressed(os.path.join(HERE, "ref_outputs.npz"), **arrays)
    print("wrote", len(arrays), "arrays")


if __name__ == "__main__":
    main()
