"""CPU: the C-ABI library loads, exports every entry point the headers
declare, and fails loudly (never silently) where no GPU is present."""
import ctypes
import os
import re

import numpy as np
import pytest

import perf_libs_sparse_b200 as pls

HEADERS = [os.path.join(pls.INCLUDE_DIR, h) for h in ("perflibs_sparse.h", "perflibs_b200.h")]


def declared_functions():
    names = set()
    for h in HEADERS:
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(perflibs_\w+)\s*\(", txt):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_the_drop_in_subset():
    names = declared_functions()
    for required in [
        "perflibs_spmat_create_csr_d", "perflibs_spmat_create_csr_s", "perflibs_spmat_create_bsr_d",
        "perflibs_spmat_create_dense_d", "perflibs_spmat_create_null", "perflibs_spmat_hint",
        "perflibs_spmv_optimize", "perflibs_spmm_optimize", "perflibs_spmv_exec_d",
        "perflibs_spmv_exec_s", "perflibs_spmm_exec_d", "perflibs_spmm_exec_s",
        "perflibs_spmat_export_csr_d", "perflibs_spmat_export_dense_d", "perflibs_spnorm_exec_d",
        "perflibs_spmat_query", "perflibs_spmat_destroy", "perflibs_spmat_print_err",
    ]:
        assert required in names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(pls.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_guard_build_exports_the_same_symbols():
    import perf_libs_sparse_b200.build as b

    if not os.path.exists(b.LIB_GUARD):
        pytest.skip("guard build not present")
    G = ctypes.CDLL(b.LIB_GUARD)
    missing = [n for n in declared_functions() if not hasattr(G, n)]
    assert not missing, missing
    G.perflibs_b200_debug_guard_violations.restype = ctypes.c_int64
    assert G.perflibs_b200_debug_guard_violations() == 0
    L = ctypes.CDLL(pls.LIB_PATH)
    L.perflibs_b200_debug_guard_violations.restype = ctypes.c_int64
    assert L.perflibs_b200_debug_guard_violations() == -1


def test_library_is_sm100a_only():
    # The fat binary carries sm_100a code only; cuobjdump is not used, the
    # build command line is the evidence.
    import perf_libs_sparse_b200.build as b

    assert b.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_enum_values_match_reference_interface():
    # include/perflibs_sparse.h:67-149 of the reference.
    assert (pls.STATUS_SUCCESS, pls.STATUS_INPUT_PARAMETER_ERROR, pls.STATUS_EXECUTION_FAILURE) == (0, 1, 2)
    assert (pls.OPERATION_NOTRANS, pls.OPERATION_TRANS, pls.OPERATION_CONJTRANS) == (300, 310, 320)
    assert (pls.INVOCATIONS_SINGLE, pls.INVOCATIONS_FEW, pls.INVOCATIONS_MANY) == (400, 410, 420)
    assert (pls.COL_MAJOR, pls.ROW_MAJOR) == (90, 91)
    assert (pls.NORM_INF, pls.NORM_FRB) == (1001, 1002)
    txt = open(HEADERS[0]).read()
    for name, val in [("PERFLIBS_SPARSE_HINT_SPMV_INVOCATIONS", 80), ("PERFLIBS_SPARSE_SCALAR_ANY", 502),
                      ("PERFLIBS_SPARSE_SPMM_STRAT_OPT_FULL_STRUCT", 603), ("PERFLIBS_SPARSE_CREATE_NOCOPY", 1)]:
        assert re.search(rf"{name}\s*=?\s*{val}\b", txt), name


def _no_gpu():
    try:
        import torch

        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="only meaningful without a GPU")
def test_fails_loudly_without_gpu():
    rp = np.array([0, 1], np.int32)
    c = np.array([0], np.int32)
    v = np.array([1.0])
    with pytest.raises(pls.PerflibsError) as e:
        pls.SpMat.csr(1, 1, rp, c, v)
    assert e.value.status == pls.STATUS_EXECUTION_FAILURE


def test_reference_driver_links_against_drop_in():
    """The reference's own benchmark driver (bench/pl_bench_sparse_x_dense.c),
    unchanged, compiles against include/perflibs_sparse.h with
    -DUSE_PERFLIBS_NAMES and links to this library: every name it uses is
    declared and exported. (Running it needs a GPU; the repository's own
    driver with the same command line runs in the GPU tests.)"""
    import subprocess

    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run(["make", "-s", "-C", os.path.join(here, "oracle"), "driver-check"],
                       capture_output=True, text=True)
    if r.returncode != 0 and "Error 77" in r.stderr:
        pytest.skip("reference sources not present")
    assert r.returncode == 0, r.stdout + r.stderr
    assert os.path.exists(os.path.join(here, "oracle", "_build", "ref_driver_on_b200"))


def test_extension_entry_points_reject_missing_arguments_on_the_host():
    """Missing handles, output pointers and paths are input errors returned
    before any device work, so they behave the same with or without a GPU;
    a tune-cache file that does not exist changes nothing."""
    L = ctypes.CDLL(pls.LIB_PATH)
    v, i32, i64, f32 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
    L.perflibs_b200_batch_create.argtypes = [v, i32, v, v, v, v, v, v, v]
    L.perflibs_b200_batch_exec.argtypes = [v, f32, f32]
    L.perflibs_b200_batch_tune.argtypes = [v, v, v]
    L.perflibs_b200_batch_set_tile.argtypes = [v, i32]
    L.perflibs_b200_batch_info.argtypes = [v, v, v, v]
    L.perflibs_b200_selector_create.argtypes = [v, i32, ctypes.c_uint64]
    L.perflibs_b200_selector_predict.argtypes = [v, v, i32, v, v]
    L.perflibs_b200_tune_cache_load.argtypes = [ctypes.c_char_p]
    L.perflibs_b200_tune_cache_save.argtypes = [ctypes.c_char_p]
    L.perflibs_b200_read_mtx.argtypes = [ctypes.c_char_p, v, v, v, v, v, v]
    L.perflibs_b200_tune_cache_size.restype = i64
    bad = pls.STATUS_INPUT_PARAMETER_ERROR
    out = v()
    assert L.perflibs_b200_batch_create(None, 1, None, None, None, None, None, None, None) == bad
    assert L.perflibs_b200_batch_create(ctypes.byref(out), 0, None, None, None, None, None, None, None) == bad
    assert L.perflibs_b200_batch_exec(None, 1.0, 0.0) == bad
    assert L.perflibs_b200_batch_tune(None, None, None) == bad
    assert L.perflibs_b200_batch_set_tile(None, 8) == bad
    assert L.perflibs_b200_batch_info(None, None, None, None) == bad
    assert L.perflibs_b200_selector_create(ctypes.byref(out), 0, 1) == bad
    assert L.perflibs_b200_selector_predict(None, None, 1, None, None) == bad
    n0 = L.perflibs_b200_tune_cache_size()
    assert L.perflibs_b200_tune_cache_load(b"/nonexistent/dir/cache.txt") == bad
    assert L.perflibs_b200_tune_cache_size() == n0
    assert L.perflibs_b200_tune_cache_save(None) == bad
    assert L.perflibs_b200_read_mtx(None, None, None, None, None, None, None) == bad
