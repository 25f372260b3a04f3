"""CPU: the launch plan of the TMA-staged diagonal-form SpMM, replayed.

tests/dia_plan_check.cpp includes the library's own planning header
(perf_libs_sparse_b200/csrc/dia_plan.hpp) and follows the kernel's work
items, tensor-map and bulk copies, barrier waits and thread reads for a
spread of matrices (27- and 7-point 3-D stencils, 5- and 9-point 2-D
stencils, bands, the 27-point 128^3 matrix of the benchmark), column counts
and element sizes: every copy must fit and be aligned, every copy must be
waited for once before its first read and never overwritten while read,
every read must hit the B row its entry needs, and every element of C must
be written exactly once. It also replays the line-patch assignment of the
diagonal-form kernel that reads B through L1 (every unit of rows computed
exactly once, for every lane count and both unit sizes)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_dia_tma_plan_replay(tmp_path):
    exe = tmp_path / "dia_plan_check"
    subprocess.run(["g++", "-O2", "-std=c++17", f"-I{os.path.join(ROOT, 'perf_libs_sparse_b200', 'csrc')}",
                    os.path.join(ROOT, "tests", "dia_plan_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("ok "), r.stdout
