"""Matrix Market input (host-only part of the library) against scipy's
reader, and the sparse x dense driver built on it."""
import os
import re
import subprocess
import zlib

import numpy as np
import pytest

import perf_libs_sparse_b200 as pls

scipy_io = pytest.importorskip("scipy.io")


def _write(path, header, size, entries):
    with open(path, "w") as f:
        f.write(header + "\n% a comment line\n")
        f.write(size + "\n")
        for e in entries:
            f.write(" ".join(str(t) for t in e) + "\n")


def _dense_from_csr(m, n, rp, c, v):
    A = np.zeros((m, n))
    for i in range(m):
        for p in range(rp[i], rp[i + 1]):
            A[i, c[p]] += v[p]
    return A


@pytest.mark.parametrize("field,sym", [("real", "general"), ("real", "symmetric"),
                                       ("real", "skew-symmetric"), ("integer", "general"),
                                       ("pattern", "general"), ("pattern", "symmetric"),
                                       ("real", "hermitian")])
def test_read_mtx_matches_scipy(tmp_path, field, sym):
    rng = np.random.default_rng(zlib.crc32(f"{field} {sym}".encode()))
    m = n = 37
    entries = set()
    while len(entries) < 120:
        r, c = int(rng.integers(1, m + 1)), int(rng.integers(1, n + 1))
        if sym != "general" and c > r:
            r, c = c, r
        if sym == "skew-symmetric" and r == c:
            continue
        entries.add((r, c))
    rows = []
    for r, c in sorted(entries):
        if field == "pattern":
            rows.append((r, c))
        elif field == "integer":
            rows.append((r, c, int(rng.integers(-9, 10))))
        else:
            rows.append((r, c, f"{rng.normal():.17g}"))
    path = tmp_path / "a.mtx"
    _write(path, f"%%MatrixMarket matrix coordinate {field} {sym}", f"{m} {n} {len(rows)}", rows)
    mm, nn, rp, c, v = pls.read_mtx(str(path))
    assert (mm, nn) == (m, n)
    # rows ordered, columns ascending within a row
    assert np.all(np.diff(rp) >= 0)
    for i in range(m):
        assert np.all(np.diff(c[rp[i]:rp[i + 1]]) >= 0)
    ref = scipy_io.mmread(str(path))
    ref = ref.toarray() if hasattr(ref, "toarray") else np.asarray(ref)
    np.testing.assert_array_equal(_dense_from_csr(m, n, rp, c, v), ref)


def test_read_mtx_keeps_duplicates_and_rectangular(tmp_path):
    path = tmp_path / "d.mtx"
    _write(path, "%%MatrixMarket matrix coordinate real general", "3 5 4",
           [(1, 5, 1.5), (3, 1, 2.0), (1, 5, -0.5), (2, 2, 4.0)])
    m, n, rp, c, v = pls.read_mtx(str(path))
    assert (m, n) == (3, 5)
    np.testing.assert_array_equal(rp, [0, 2, 3, 4])
    np.testing.assert_array_equal(c, [4, 4, 1, 0])
    np.testing.assert_array_equal(v, [1.5, -0.5, 4.0, 2.0])  # equal positions in file order


@pytest.mark.parametrize("text", [
    "%%MatrixMarket matrix coordinate complex general\n2 2 1\n1 1 1 0\n",
    "%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n",
    "%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1.0\n",
    "not a matrix market file\n",
])
def test_read_mtx_rejects_bad_files(tmp_path, text):
    path = tmp_path / "bad.mtx"
    path.write_text(text)
    with pytest.raises(pls.PerflibsError):
        pls.read_mtx(str(path))
    with pytest.raises(pls.PerflibsError):
        pls.read_mtx(str(tmp_path / "missing.mtx"))


@pytest.mark.gpu
def test_driver_runs_on_laplacian(tmp_path):
    """The driver reads the file, runs spmm_optimize + 10 spmm_exec_d on the
    GPU and prints the reference driver's four lines."""
    from perf_libs_sparse_b200 import workloads as W

    m, n, rp, c, v = W.laplacian_2d(64)
    path = tmp_path / "lap.mtx"
    ent = [(i + 1, int(c[p]) + 1, v[p]) for i in range(m) for p in range(rp[i], rp[i + 1])]
    _write(path, "%%MatrixMarket matrix coordinate real general", f"{m} {n} {len(ent)}", ent)
    exe = os.path.join(os.path.dirname(pls.__file__), "bench_sparse_x_dense")
    out = subprocess.run([exe, str(path)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    assert lines[0] == f"A: {m} x {n} nnz={len(ent)}"
    assert lines[1] == f"B: {n} x 1024" and lines[2] == f"C: {m} x 1024"
    assert re.fullmatch(r"iters=10 total_s=[0-9.]+ avg_s=[0-9.]+", lines[3])
