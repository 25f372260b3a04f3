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
    # more entries than any host can hold: the allocation fails inside the
    # library and comes back as a status, not as an exception
    "%%MatrixMarket matrix coordinate real general\n2 2 4000000000000000000\n1 1 1.0\n",
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


@pytest.mark.gpu
def test_reference_driver_runs_on_gpu(tmp_path):
    """The reference's own benchmark driver (bench/pl_bench_sparse_x_dense.c,
    unchanged, compiled against include/perflibs_sparse.h and linked to this
    library by `make -C oracle driver-check`) runs on the GPU: it reads a
    Matrix Market file, fills B (n x 1024) from srand(1) / rand(), and runs
    spmm_optimize + 10 spmm_exec_d. A preloaded tap (tests/ref_driver_tap.c)
    writes the C of each exec; the last one must equal the FP64 oracle's
    A*B within 1e-12 (scaled per element), with B rebuilt here from the same
    C library's rand()."""
    import ctypes

    import oracle
    from perf_libs_sparse_b200 import workloads as W
    from tests.conftest import spmm_row_err

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "oracle", "_build", "ref_driver_on_b200")
    if not os.path.exists(exe):
        pytest.skip("the reference driver was not built (make -C oracle driver-check)")
    tap = tmp_path / "tap.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-O2", f"-I{os.path.join(root, 'include')}",
                    os.path.join(root, "tests", "ref_driver_tap.c"), "-o", str(tap), "-ldl"], check=True)
    rng = np.random.default_rng(31)
    m, n = 300, 260
    rp, c, v = W.random_csr(m, n, 20, rng, empty_frac=0.1)
    path = tmp_path / "r.mtx"
    ent = [(i + 1, int(c[p]) + 1, f"{v[p]:.17g}") for i in range(m) for p in range(rp[i], rp[i + 1])]
    _write(path, "%%MatrixMarket matrix coordinate real general", f"{m} {n} {len(ent)}", ent)
    out_c = tmp_path / "c.bin"
    env = dict(os.environ, LD_PRELOAD=str(tap), PERFLIBS_TAP_C=str(out_c),
               LD_LIBRARY_PATH=os.path.dirname(pls.__file__) + os.pathsep + os.environ.get("LD_LIBRARY_PATH", ""))
    r = subprocess.run([exe, str(path)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    assert lines[0] == f"A: {m} x {n} nnz={len(ent)}"
    assert lines[2] == f"C: {m} x 1024"
    assert re.fullmatch(r"iters=10 total_s=[0-9.]+ avg_s=[0-9.]+", lines[3])
    raw = out_c.read_bytes()
    mm, nn = np.frombuffer(raw[:8], np.int32)
    assert (mm, nn) == (m, 1024)
    got = np.frombuffer(raw[8:], np.float64).reshape(m, 1024)
    libc = ctypes.CDLL(None)
    libc.rand.restype = ctypes.c_int
    libc.srand(1)
    rand_max = 2147483647.0  # glibc RAND_MAX
    B = np.array([2.0 * libc.rand() / rand_max - 1.0 for _ in range(n * 1024)]).reshape(n, 1024)
    ref = oracle.csr_spmm(rp, c, v, B, 1024)
    assert spmm_row_err(got, ref, rp, c, v, B, 1.0) <= 1e-12
