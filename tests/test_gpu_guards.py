"""The GPU parity tests again, under the guard build of the library: every
device buffer the library allocates is followed by a guard of 0xFF bytes,
checked when the buffer is freed. A kernel writing past a buffer's end fails
the run (the session check in conftest.py); one reading past it reads NaN
into a result, which the parity assertions catch. This stands in for
compute-sanitizer's memcheck, which is not available on every machine."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GUARD_LIB = os.path.join(ROOT, "perf_libs_sparse_b200", "libplsparse_b200_guard.so")
SUITES = ["test_gpu_spmv.py", "test_gpu_edges.py", "test_gpu_spmm.py", "test_gpu_batch.py",
          "test_gpu_convert.py"]


def test_parity_suites_under_guard_build():
    from perf_libs_sparse_b200 import build as b

    assert b.build(guards=True) == GUARD_LIB  # rebuilt only when older than its sources
    env = dict(os.environ, PERFLIBS_B200_LIBRARY=GUARD_LIB)
    r = subprocess.run(
        [sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider",
         *[os.path.join(ROOT, "tests", f) for f in SUITES]],
        cwd=ROOT, env=env, capture_output=True, text=True, timeout=1800)
    tail = (r.stdout + r.stderr)[-3000:]
    assert r.returncode == 0, tail
    assert "a write past a device buffer" not in r.stderr, tail
