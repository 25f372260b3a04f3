"""Build libplsparse_b200.so in-tree for sm_100a.

Compiles every ``csrc/*.cu`` with nvcc for ``compute_100a``/``sm_100a`` (no
other architecture), in parallel, and links the C-ABI shared library next to
this file. The CUDA runtime is linked statically (nvcc's default), so the
library only needs the driver at run time.

The guard build (``--guards``) is the same library with -DPLS_DEBUG_GUARDS:
every device buffer is followed by a guard region checked when the buffer is
freed. It goes to libplsparse_b200_guard.so, beside the regular one, and is
loaded instead of it when PERFLIBS_B200_LIBRARY names it.

Usage: python -m perf_libs_sparse_b200.build [--verbose-ptxas] [--force] [--guards]
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libplsparse_b200.so")
OBJ_GUARD = os.path.join(HERE, "_build_guard")
LIB_GUARD = os.path.join(HERE, "libplsparse_b200_guard.so")
DRIVERS = os.path.join(HERE, "drivers")
BENCH_DRIVER = os.path.join(HERE, "bench_sparse_x_dense")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-DNDEBUG",
          "--expt-relaxed-constexpr", f"-I{os.path.join(ROOT, 'include')}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: str, verbose_ptxas: bool, guards: bool = False) -> tuple[str, str]:
    obj = os.path.join(OBJ_GUARD if guards else OBJ, os.path.basename(src).replace(".cu", ".o"))
    cmd = [nvcc(), *ARCH, *CFLAGS, *(["-DPLS_DEBUG_GUARDS"] if guards else []), "-c", src,
           "-o", obj]
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def stale(guards: bool = False) -> bool:
    lib = LIB_GUARD if guards else LIB
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    if not guards and not os.path.exists(BENCH_DRIVER):
        return True
    for d in (CSRC, DRIVERS, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if os.path.getmtime(os.path.join(d, f)) > t:
                return True
    return False


def build(verbose_ptxas: bool = False, force: bool = False, guards: bool = False) -> str:
    lib = LIB_GUARD if guards else LIB
    if not force and not stale(guards):
        return lib
    os.makedirs(OBJ_GUARD if guards else OBJ, exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose_ptxas, guards), srcs))
    if verbose_ptxas:
        for obj, log in results:
            sys.stderr.write(log)
    objs = [o for o, _ in results]
    tmp = lib + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-Xlinker", f"-soname={os.path.basename(lib)}", "-o", tmp,
           *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib)
    if not guards:
        _build_driver()
    return lib


def _build_driver() -> None:
    """The Matrix Market SpMM driver (drivers/bench_sparse_x_dense.c), a
    plain C program on the drop-in interface, linked to the library next to
    it (rpath $ORIGIN)."""
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        raise RuntimeError("no C compiler for the driver")
    cmd = [cc, "-O2", "-std=c11", f"-I{os.path.join(ROOT, 'include')}",
           os.path.join(DRIVERS, "bench_sparse_x_dense.c"), LIB, "-Wl,-rpath,$ORIGIN", "-lm",
           "-o", BENCH_DRIVER]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"driver build failed:\n{r.stdout}\n{r.stderr}")


if __name__ == "__main__":
    print(build(verbose_ptxas="--verbose-ptxas" in sys.argv, force="--force" in sys.argv,
                guards="--guards" in sys.argv))
