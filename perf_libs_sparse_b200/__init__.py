"""Python mirror of the perflibs_sparse C interface, over libplsparse_b200.so.

The product is the C-ABI shared library built from ``csrc/`` (declared in
``include/perflibs_sparse.h`` and ``include/perflibs_b200.h``). This module
binds it with ctypes so that tests and benchmarks drive exactly the entry
points a C caller links against: create -> hint -> optimize -> exec ->
export -> destroy, with the reference's enum values and status codes.

There is no fallback: importing works without a GPU (for symbol checks), but
any call that needs the device raises ``PerflibsError`` when the CUDA
library or the device is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# PERFLIBS_B200_LIBRARY selects another build of the library (the guard
# build, libplsparse_b200_guard.so, for instance).
LIB_PATH = os.environ.get("PERFLIBS_B200_LIBRARY") or os.path.join(HERE, "libplsparse_b200.so")
ROOT = os.path.dirname(HERE)
INCLUDE_DIR = os.path.join(ROOT, "include")

# ---------------------------------------------------------------- enums
# Values of the reference interface (include/perflibs_sparse.h:67-149).
STATUS_SUCCESS = 0
STATUS_INPUT_PARAMETER_ERROR = 1
STATUS_EXECUTION_FAILURE = 2

HINT_STRUCTURE = 50
HINT_SPMV_OPERATION = 60
HINT_SPMM_OPERATION = 61
HINT_MEMORY = 70
HINT_SPMV_INVOCATIONS = 80
HINT_SPMM_INVOCATIONS = 81

COL_MAJOR = 90
ROW_MAJOR = 91

STRUCTURE_UNSTRUCTURED = 101
OPERATION_NOTRANS = 300
OPERATION_TRANS = 310
OPERATION_CONJTRANS = 320
INVOCATIONS_SINGLE = 400
INVOCATIONS_FEW = 410
INVOCATIONS_MANY = 420
SCALAR_ONE = 500
SCALAR_ZERO = 501
SCALAR_ANY = 502
NORM_INF = 1001
NORM_FRB = 1002
CREATE_NOCOPY = 1

# Extensions (include/perflibs_b200.h).
STORAGE_NATIVE, STORAGE_FP32, STORAGE_BF16 = 0, 1, 2
TUNE_EXHAUSTIVE, TUNE_SELECTOR, TUNE_NONE = 0, 1, 2
KIND_CSR, KIND_SELL, KIND_CSR_SPLIT = 0, 1, 2


class PerflibsError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: status {status}")
        self.status = status


_lib = None


def lib():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise PerflibsError(STATUS_EXECUTION_FAILURE,
                                f"{LIB_PATH} is missing; run perf_libs_sparse_b200.build")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, d, f, i = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_float, C.c_int
        sig = {
            "perflibs_spmat_create_csr_s": [vp, i32, i32, vp, vp, vp, i32],
            "perflibs_spmat_create_csr_d": [vp, i32, i32, vp, vp, vp, i32],
            "perflibs_spmat_create_dense_s": [vp, i, i32, i32, i32, vp, i32],
            "perflibs_spmat_create_dense_d": [vp, i, i32, i32, i32, vp, i32],
            "perflibs_spmat_create_bsr_s": [vp, i, i32, i32, i32, vp, vp, vp, i32],
            "perflibs_spmat_create_bsr_d": [vp, i, i32, i32, i32, vp, vp, vp, i32],
            "perflibs_spmat_create_csc_s": [vp, i32, i32, vp, vp, vp, i32],
            "perflibs_spmat_create_csc_d": [vp, i32, i32, vp, vp, vp, i32],
            "perflibs_spmat_create_coo_s": [vp, i32, i32, i32, vp, vp, vp, i32],
            "perflibs_spmat_create_coo_d": [vp, i32, i32, i32, vp, vp, vp, i32],
            "perflibs_spmat_create_null": [i32, i32],
            "perflibs_spmat_create_identity": [i32],
            "perflibs_spmat_destroy": [vp],
            "perflibs_spmat_query": [vp, vp, vp, vp, vp],
            "perflibs_spmat_hint": [vp, i, i],
            "perflibs_spmv_optimize": [vp],
            "perflibs_spmm_optimize": [i, i, i, vp, vp, i, vp],
            "perflibs_spmv_exec_s": [i, f, vp, vp, f, vp],
            "perflibs_spmv_exec_d": [i, d, vp, vp, d, vp],
            "perflibs_spmm_exec_s": [i, i, f, vp, vp, f, vp],
            "perflibs_spmm_exec_d": [i, i, d, vp, vp, d, vp],
            "perflibs_spmat_update_s": [vp, i32, vp, vp, vp],
            "perflibs_spmat_update_d": [vp, i32, vp, vp, vp],
            "perflibs_spmat_export_csr_s": [vp, i32, vp, vp, vp, vp, vp],
            "perflibs_spmat_export_csr_d": [vp, i32, vp, vp, vp, vp, vp],
            "perflibs_spmat_export_dense_s": [vp, i, vp, vp, vp],
            "perflibs_spmat_export_dense_d": [vp, i, vp, vp, vp],
            "perflibs_spnorm_exec_s": [vp, i, vp],
            "perflibs_spnorm_exec_d": [vp, i, vp],
            "perflibs_spmat_print_err": [vp],
            "perflibs_b200_spmat_get_error": [vp, vp, vp, vp, i32],
            "perflibs_b200_spmat_spmm_info": [vp, vp, vp, vp, vp, vp, vp],
            "perflibs_b200_spmat_set_spmm_path": [vp, i32],
            "perflibs_b200_spmat_set_host_bands": [vp, i32],
            "perflibs_b200_spmat_create_csr_d_dev": [vp, i32, i32, vp, vp, vp, vp],
            "perflibs_b200_spmat_host_bands_used": [vp, vp],
            "perflibs_b200_spmat_tune_source": [vp, vp],
            "perflibs_b200_tune_cache_save": [C.c_char_p],
            "perflibs_b200_tune_cache_load": [C.c_char_p],
            "perflibs_b200_tune_cache_clear": [],
            "perflibs_b200_read_mtx": [C.c_char_p, vp, vp, vp, vp, vp, vp],
            "perflibs_b200_testing_stage_fault": [i32, i32],
            "perflibs_b200_spmv_exec_d_dev": [i, d, vp, vp, d, vp, vp],
            "perflibs_b200_spmv_exec_s_dev": [i, f, vp, vp, f, vp, vp],
            "perflibs_b200_spmm_exec_d_dev": [d, vp, vp, i64, i32, d, vp, i64, vp],
            "perflibs_b200_spmm_exec_s_dev": [f, vp, vp, i64, i32, f, vp, i64, vp],
            "perflibs_b200_spmat_set_storage": [vp, i],
            "perflibs_b200_spmat_set_tuner": [vp, i],
            "perflibs_b200_spmat_force_config": [vp, i, i, i, i],
            "perflibs_b200_spmat_get_config": [vp, vp, vp, vp, vp, vp],
            "perflibs_b200_spmat_tune_table": [vp, i32, vp, vp, vp, vp],
            "perflibs_b200_spmat_exec_info": [vp, vp, vp, vp],
            "perflibs_b200_spmat_export_sell": [vp, vp, vp, vp, vp, vp, vp, vp, vp],
            "perflibs_b200_spmat_build_sell": [vp, i, i],
            "perflibs_b200_spmat_set_stream": [vp, vp],
            "perflibs_b200_spmat_csr_to_bsr": [vp, i32, i, vp],
            "perflibs_b200_spmat_export_bsr_d": [vp, vp, vp, vp, vp, vp],
            "perflibs_b200_device_info": [vp, vp, vp],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        L.perflibs_spmat_create_null.restype = vp
        L.perflibs_spmat_create_identity.restype = vp
        L.perflibs_spmat_print_err.restype = None
        L.perflibs_b200_version.restype = C.c_char_p
        L.perflibs_b200_tune_cache_size.argtypes = []
        L.perflibs_b200_tune_cache_size.restype = C.c_int64
        L.perflibs_b200_debug_guard_violations.argtypes = []
        L.perflibs_b200_debug_guard_violations.restype = C.c_int64
        _lib = L
    return _lib


_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(st: int, what: str):
    if st != STATUS_SUCCESS:
        raise PerflibsError(st, what)


def device_info():
    sm, l2, dev = C.c_int32(), C.c_int64(), C.c_int32()
    _check(lib().perflibs_b200_device_info(C.byref(sm), C.byref(l2), C.byref(dev)), "device_info")
    return {"sm_count": sm.value, "l2_bytes": l2.value, "device": dev.value}


class SpMat:
    """An owned perflibs_spmat_t handle."""

    def __init__(self, handle, dtype):
        self.h = C.c_void_p(handle) if not isinstance(handle, C.c_void_p) else handle
        self.dtype = np.dtype(dtype)

    # -------------------------------------------------------- creation
    @staticmethod
    def csr(m, n, row_ptr, col, vals, flags=0, check=True):
        vals = np.ascontiguousarray(vals)
        row_ptr = np.ascontiguousarray(row_ptr, np.int32)
        col = np.ascontiguousarray(col, np.int32)
        h = C.c_void_p()
        fn = lib().perflibs_spmat_create_csr_s if vals.dtype == np.float32 else lib().perflibs_spmat_create_csr_d
        st = fn(C.byref(h), m, n, _p(row_ptr), _p(col), _p(vals), flags)
        M = SpMat(h, vals.dtype)
        M.status = st
        if check:
            _check(st, "create_csr")
        return M

    @staticmethod
    def csr_dev(m, n, row_ptr_ptr: int, col_ptr: int, vals_ptr: int, stream: int = 0):
        """FP64 CSR handle from arrays already on the device (int32 row
        pointers and columns, double values; copied), e.g. torch tensors'
        data_ptr()."""
        h = C.c_void_p()
        _check(lib().perflibs_b200_spmat_create_csr_d_dev(
            C.byref(h), m, n, C.c_void_p(row_ptr_ptr), C.c_void_p(col_ptr), C.c_void_p(vals_ptr),
            C.c_void_p(stream)), "create_csr_d_dev")
        return SpMat(h, np.float64)

    @staticmethod
    def coo(m, n, row, col, vals, flags=0, check=True):
        """COO input (0-based, any order, duplicates allowed); the library
        converts it to CSR on the device."""
        vals = np.ascontiguousarray(vals)
        row = np.ascontiguousarray(row, np.int32)
        col = np.ascontiguousarray(col, np.int32)
        h = C.c_void_p()
        fn = lib().perflibs_spmat_create_coo_s if vals.dtype == np.float32 else lib().perflibs_spmat_create_coo_d
        st = fn(C.byref(h), m, n, len(vals), _p(row), _p(col), _p(vals), flags)
        M = SpMat(h, vals.dtype)
        M.status = st
        if check:
            _check(st, "create_coo")
        return M

    @staticmethod
    def csc(m, n, row_indx, col_ptr, vals, flags=0, check=True):
        """CSC input (0- or 1-based, as col_ptr[0] says)."""
        vals = np.ascontiguousarray(vals)
        row_indx = np.ascontiguousarray(row_indx, np.int32)
        col_ptr = np.ascontiguousarray(col_ptr, np.int32)
        h = C.c_void_p()
        fn = lib().perflibs_spmat_create_csc_s if vals.dtype == np.float32 else lib().perflibs_spmat_create_csc_d
        st = fn(C.byref(h), m, n, _p(row_indx), _p(col_ptr), _p(vals), flags)
        M = SpMat(h, vals.dtype)
        M.status = st
        if check:
            _check(st, "create_csc")
        return M

    @staticmethod
    def bsr(layout, m, n, bs, row_ptr, col, vals, flags=0, check=True):
        vals = np.ascontiguousarray(vals)
        row_ptr = np.ascontiguousarray(row_ptr, np.int32)
        col = np.ascontiguousarray(col, np.int32)
        h = C.c_void_p()
        fn = lib().perflibs_spmat_create_bsr_s if vals.dtype == np.float32 else lib().perflibs_spmat_create_bsr_d
        st = fn(C.byref(h), layout, m, n, bs, _p(row_ptr), _p(col), _p(vals), flags)
        M = SpMat(h, vals.dtype)
        M.status = st
        if check:
            _check(st, "create_bsr")
        return M

    @staticmethod
    def dense(layout, m, n, lda, vals, flags=0, check=True):
        vals = np.ascontiguousarray(vals)
        h = C.c_void_p()
        fn = lib().perflibs_spmat_create_dense_s if vals.dtype == np.float32 else lib().perflibs_spmat_create_dense_d
        st = fn(C.byref(h), layout, m, n, lda, _p(vals), flags)
        M = SpMat(h, vals.dtype)
        M.status = st
        if check:
            _check(st, "create_dense")
        return M

    @staticmethod
    def null(m, n, dtype=np.float64):
        h = lib().perflibs_spmat_create_null(m, n)
        if not h:
            raise PerflibsError(STATUS_INPUT_PARAMETER_ERROR, "create_null")
        return SpMat(h, dtype)

    @staticmethod
    def identity(n, dtype=np.float64):
        h = lib().perflibs_spmat_create_identity(n)
        if not h:
            raise PerflibsError(STATUS_INPUT_PARAMETER_ERROR, "create_identity")
        return SpMat(h, dtype)

    # --------------------------------------------------------- control
    def hint(self, hint, value):
        return lib().perflibs_spmat_hint(self.h, hint, value)

    def optimize(self):
        return lib().perflibs_spmv_optimize(self.h)

    def query(self):
        b, m, n, z = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        _check(lib().perflibs_spmat_query(self.h, C.byref(b), C.byref(m), C.byref(n), C.byref(z)), "query")
        return b.value, m.value, n.value, z.value

    def set_storage(self, mode):
        return lib().perflibs_b200_spmat_set_storage(self.h, mode)

    def set_tuner(self, mode):
        return lib().perflibs_b200_spmat_set_tuner(self.h, mode)

    def force_config(self, kind, C_=0, sigma=0, tpr=0):
        return lib().perflibs_b200_spmat_force_config(self.h, kind, C_, sigma, tpr)

    def build_sell(self, C_, sigma):
        return lib().perflibs_b200_spmat_build_sell(self.h, C_, sigma)

    def set_stream(self, stream_ptr: int):
        return lib().perflibs_b200_spmat_set_stream(self.h, C.c_void_p(stream_ptr))

    def config(self):
        k, c, s, t, b = (C.c_int() for _ in range(5))
        _check(lib().perflibs_b200_spmat_get_config(self.h, C.byref(k), C.byref(c), C.byref(s),
                                                    C.byref(t), C.byref(b)), "get_config")
        return {"kind": k.value, "C": c.value, "sigma": s.value, "tpr": t.value, "col_bytes": b.value}

    def exec_info(self):
        k, it, sp = C.c_int32(), C.c_int64(), C.c_int64()
        _check(lib().perflibs_b200_spmat_exec_info(self.h, C.byref(k), C.byref(it), C.byref(sp)),
               "exec_info")
        return {"kernels_per_spmv": k.value, "n_items": it.value, "n_split": sp.value}

    def tune_table(self, with_beta=False):
        cnt = C.c_int32()
        lib().perflibs_b200_spmat_tune_table(self.h, 0, None, None, None, C.byref(cnt))
        n = cnt.value
        cfg = np.zeros((max(n, 1), 4), np.int32)
        ms = np.zeros(max(n, 1))
        beta = np.zeros(max(n, 1))
        lib().perflibs_b200_spmat_tune_table(self.h, n, _p(cfg), _p(ms), _p(beta), C.byref(cnt))
        if with_beta:
            return cfg[:n], ms[:n], beta[:n]
        return cfg[:n], ms[:n]

    # -------------------------------------------------------- execution
    def spmv(self, x, y=None, alpha=1.0, beta=0.0, trans=OPERATION_NOTRANS, check=True):
        """Host-pointer exec (the drop-in perflibs_spmv_exec_{s,d})."""
        x = np.ascontiguousarray(x, self.dtype)
        _, m, n, _ = self.query()
        ylen = m if trans == OPERATION_NOTRANS else n
        y = np.zeros(ylen, self.dtype) if y is None else y
        fn = lib().perflibs_spmv_exec_s if self.dtype == np.float32 else lib().perflibs_spmv_exec_d
        st = fn(trans, alpha, self.h, _p(x), beta, _p(y))
        if check:
            _check(st, "spmv_exec")
        return y if check else (st, y)

    def spmv_dev(self, x_ptr: int, y_ptr: int, alpha=1.0, beta=0.0, stream: int = 0,
                 trans=OPERATION_NOTRANS):
        fn = lib().perflibs_b200_spmv_exec_s_dev if self.dtype == np.float32 else lib().perflibs_b200_spmv_exec_d_dev
        _check(fn(trans, alpha, self.h, C.c_void_p(x_ptr), beta, C.c_void_p(y_ptr),
                  C.c_void_p(stream)), "spmv_exec_dev")

    def spmm_dev(self, B_ptr: int, ldb: int, k: int, C_ptr: int, ldc: int, alpha=1.0, beta=0.0,
                 stream: int = 0):
        fn = lib().perflibs_b200_spmm_exec_s_dev if self.dtype == np.float32 else lib().perflibs_b200_spmm_exec_d_dev
        _check(fn(alpha, self.h, C.c_void_p(B_ptr), ldb, k, beta, C.c_void_p(C_ptr), ldc,
                  C.c_void_p(stream)), "spmm_exec_dev")

    def update(self, rows, cols, vals):
        rows = np.ascontiguousarray(rows, np.int32)
        cols = np.ascontiguousarray(cols, np.int32)
        vals = np.ascontiguousarray(vals, self.dtype)
        fn = lib().perflibs_spmat_update_s if self.dtype == np.float32 else lib().perflibs_spmat_update_d
        return fn(self.h, len(rows), _p(rows), _p(cols), _p(vals))

    def norm(self, kind=NORM_INF):
        if self.dtype == np.float32:
            r = C.c_float()
            st = lib().perflibs_spnorm_exec_s(self.h, kind, C.byref(r))
        else:
            r = C.c_double()
            st = lib().perflibs_spnorm_exec_d(self.h, kind, C.byref(r))
        _check(st, "spnorm")
        return r.value

    # ----------------------------------------------------------- export
    def export_csr(self, index_base=0):
        m, n = C.c_int32(), C.c_int32()
        rp, ci, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
        fn = lib().perflibs_spmat_export_csr_s if self.dtype == np.float32 else lib().perflibs_spmat_export_csr_d
        _check(fn(self.h, index_base, C.byref(m), C.byref(n), C.byref(rp), C.byref(ci), C.byref(v)),
               "export_csr")
        try:
            M = m.value
            rpa = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_int32)), (M + 1,)).copy()
            nnz = int(rpa[-1] - index_base)
            cia = np.ctypeslib.as_array(C.cast(ci, C.POINTER(C.c_int32)), (max(nnz, 1),))[:nnz].copy()
            ct = C.c_float if self.dtype == np.float32 else C.c_double
            va = np.ctypeslib.as_array(C.cast(v, C.POINTER(ct)), (max(nnz, 1),))[:nnz].copy()
        finally:
            for p in (rp, ci, v):
                _libc.free(p)
        return m.value, n.value, rpa, cia, va

    def export_dense(self, layout=ROW_MAJOR):
        m, n = C.c_int32(), C.c_int32()
        v = C.c_void_p()
        fn = lib().perflibs_spmat_export_dense_s if self.dtype == np.float32 else lib().perflibs_spmat_export_dense_d
        _check(fn(self.h, layout, C.byref(m), C.byref(n), C.byref(v)), "export_dense")
        try:
            ct = C.c_float if self.dtype == np.float32 else C.c_double
            a = np.ctypeslib.as_array(C.cast(v, C.POINTER(ct)), (m.value * n.value,)).copy()
        finally:
            _libc.free(v)
        if layout == ROW_MAJOR:
            return a.reshape(m.value, n.value)
        return a.reshape(n.value, m.value).T

    def export_sell(self, vals_dtype=np.float64):
        info = np.zeros(7, np.int64)
        _check(lib().perflibs_b200_spmat_export_sell(self.h, _p(info), None, None, None, None, None,
                                                     None, None), "export_sell")
        nC, Cc, sg, nb, nfull, ntidy, size = (int(v) for v in info)
        cs = np.zeros(max(nC, 1), np.int64)
        cl = np.zeros(max(nC, 1), np.int64)
        cm = np.zeros(max(nC, 1), np.int64)
        p2i = np.zeros(max(nC * Cc, 1), np.int64)
        i2p = np.zeros(max(nC * Cc, 1), np.int64)
        v = np.zeros(max(size, 1), vals_dtype)
        raw = np.zeros(max(size * nb, 1), np.uint8)
        _check(lib().perflibs_b200_spmat_export_sell(self.h, _p(info), _p(cs), _p(cl), _p(cm), _p(p2i),
                                                     _p(i2p), _p(v), _p(raw)), "export_sell")
        odt = {1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}[nb]
        return dict(nC=nC, C=Cc, sigma=sg, size=size, cs=cs[:nC], cl=cl[:nC], col_min=cm[:nC],
                    permd2in=p2i[: nC * Cc], in2permd=i2p[: nC * Cc], vals=v[:size],
                    offsets=raw[: size * nb].view(odt).astype(np.int64), col_bytes=nb,
                    n_full_chunks=nfull, ntidyup=ntidy)

    def to_bsr(self, bs, layout=ROW_MAJOR):
        h = C.c_void_p()
        _check(lib().perflibs_b200_spmat_csr_to_bsr(self.h, bs, layout, C.byref(h)), "csr_to_bsr")
        return SpMat(h, self.dtype)

    def export_bsr(self):
        bs, nnzb = C.c_int32(), C.c_int32()
        rp, ci, v = C.c_void_p(), C.c_void_p(), C.c_void_p()
        _check(lib().perflibs_b200_spmat_export_bsr_d(self.h, C.byref(bs), C.byref(nnzb), C.byref(rp),
                                                      C.byref(ci), C.byref(v)), "export_bsr")
        _, m, _, _ = self.query()
        try:
            mb = m // bs.value
            rpa = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_int32)), (mb + 1,)).copy()
            k = nnzb.value
            cia = np.ctypeslib.as_array(C.cast(ci, C.POINTER(C.c_int32)), (max(k, 1),))[:k].copy()
            e = k * bs.value * bs.value
            va = np.ctypeslib.as_array(C.cast(v, C.POINTER(C.c_double)), (max(e, 1),))[:e].copy()
        finally:
            for p in (rp, ci, v):
                _libc.free(p)
        return bs.value, rpa, cia, va

    def print_err(self):
        lib().perflibs_spmat_print_err(self.h)

    def error(self):
        """(status, argument position, message) of the handle's last error."""
        t, c = C.c_int32(), C.c_int32()
        buf = C.create_string_buffer(512)
        lib().perflibs_b200_spmat_get_error(self.h, C.byref(t), C.byref(c), buf, 512)
        return t.value, c.value, buf.value.decode(errors="replace")

    def error_code(self):
        return self.error()[1]

    def spmm_info(self):
        """SpMM plan: tile_rows (0 = no staged tiles), staged_rows, runs,
        path of the last SpMM (1 staged, 0 row group, 2 row group with shared
        entries, 3 diagonal form, 4 diagonal form with TMA-staged B, 5 BSR on
        the tensor cores, 6 BSR FMA kernel, -1 none) and the two
        timings of the measured choice (ms, 0 when not measured)."""
        r, u, n, pth = C.c_int32(), C.c_int64(), C.c_int64(), C.c_int32()
        ms_s, ms_r = C.c_float(), C.c_float()
        _check(lib().perflibs_b200_spmat_spmm_info(self.h, C.byref(r), C.byref(u), C.byref(n),
                                                   C.byref(pth), C.byref(ms_s), C.byref(ms_r)),
               "spmm_info")
        return {"tile_rows": r.value, "staged_rows": u.value, "runs": n.value, "path": pth.value,
                "ms_staged": ms_s.value, "ms_rows": ms_r.value}

    def set_spmm_path(self, path):
        """-1 measured choice (default), 0 row-group kernel, 1 staged kernel,
        2 row-group kernel with shared entries, 3 diagonal-form kernel, 4
        diagonal form with TMA-staged B, 5 BSR on the tensor cores (each where
        it applies; otherwise the row-group kernel runs, or for 4 the diagonal
        form when it applies, for 5 the BSR FMA kernel)."""
        _check(lib().perflibs_b200_spmat_set_spmm_path(self.h, path), "set_spmm_path")

    def set_host_bands(self, n_bands):
        """Row bands of host-buffer SpMV: 0 by size (default), 1 none, 2..64 that many."""
        _check(lib().perflibs_b200_spmat_set_host_bands(self.h, n_bands), "set_host_bands")

    def tune_source(self):
        """How the active SpMV configuration was chosen (TUNE_SOURCE_*)."""
        r = C.c_int32()
        _check(lib().perflibs_b200_spmat_tune_source(self.h, C.byref(r)), "tune_source")
        return r.value

    def host_bands_used(self):
        """Bands the last host-buffer SpMV ran in (0 = one launch)."""
        r = C.c_int32()
        _check(lib().perflibs_b200_spmat_host_bands_used(self.h, C.byref(r)), "host_bands_used")
        return r.value

    def destroy(self):
        if self.h is not None and self.h.value:
            lib().perflibs_spmat_destroy(self.h)
        self.h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class Batch:
    """perflibs_b200_batch_t: many independent FP32 SpMMs in one persistent
    launch. B and C are lists of device pointers (int) with their leading
    dimensions; the handles must stay unchanged while the batch exists."""

    def __init__(self, mats, ks, Bptrs, ldbs, Cptrs, ldcs, stream: int = 0):
        L = lib()
        vp = C.c_void_p
        for name, args in {"perflibs_b200_batch_create": [vp, C.c_int32, vp, vp, vp, vp, vp, vp, vp],
                           "perflibs_b200_batch_set_tile": [vp, C.c_int32],
                           "perflibs_b200_batch_tune": [vp, vp, vp],
                           "perflibs_b200_batch_exec": [vp, C.c_float, C.c_float],
                           "perflibs_b200_batch_info": [vp, vp, vp, vp],
                           "perflibs_b200_batch_set_staging": [vp, C.c_int32],
                           "perflibs_b200_batch_stage_info": [vp, vp, vp],
                           "perflibs_b200_batch_destroy": [vp]}.items():
            getattr(L, name).argtypes = args
            getattr(L, name).restype = C.c_int
        n = len(mats)
        self._mats = list(mats)  # keep the handles alive
        hs = (C.c_void_p * n)(*[m.h.value for m in mats])
        k = np.ascontiguousarray(ks, np.int32)
        ldb = np.ascontiguousarray(ldbs, np.int64)
        ldc = np.ascontiguousarray(ldcs, np.int64)
        bp = (C.c_void_p * n)(*Bptrs)
        cp = (C.c_void_p * n)(*Cptrs)
        self.h = C.c_void_p()
        _check(L.perflibs_b200_batch_create(C.byref(self.h), n, hs, _p(k), bp, _p(ldb), cp, _p(ldc),
                                            C.c_void_p(stream)), "batch_create")

    def tune(self):
        t, ms = C.c_int32(), C.c_float()
        _check(lib().perflibs_b200_batch_tune(self.h, C.byref(t), C.byref(ms)), "batch_tune")
        return t.value, ms.value

    def set_tile(self, rows):
        _check(lib().perflibs_b200_batch_set_tile(self.h, rows), "batch_set_tile")

    def exec(self, alpha=1.0, beta=0.0):
        _check(lib().perflibs_b200_batch_exec(self.h, alpha, beta), "batch_exec")

    def info(self):
        n, l, t = C.c_int64(), C.c_int32(), C.c_int32()
        _check(lib().perflibs_b200_batch_info(self.h, C.byref(n), C.byref(l), C.byref(t)), "batch_info")
        return {"n_items": n.value, "launches": l.value, "tile": t.value}

    def set_staging(self, on):
        """Run the staged (shared-memory window) items (True) or send every
        row to the per-warp items (False)."""
        _check(lib().perflibs_b200_batch_set_staging(self.h, 1 if on else 0), "batch_set_staging")

    def stage_info(self):
        """{'staged_items': built at creation, 'staging': whether they run}."""
        n, on = C.c_int64(), C.c_int32()
        _check(lib().perflibs_b200_batch_stage_info(self.h, C.byref(n), C.byref(on)), "batch_stage_info")
        return {"staged_items": n.value, "staging": bool(on.value)}

    def destroy(self):
        if self.h is not None and self.h.value:
            lib().perflibs_b200_batch_destroy(self.h)
        self.h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


# Autotune cache (checkpoint / resume of the exhaustive tuner).
TUNE_SOURCE_NONE, TUNE_SOURCE_TIMED, TUNE_SOURCE_CACHE, TUNE_SOURCE_SELECTOR, TUNE_SOURCE_FORCED = range(5)


def tune_cache_save(path):
    _check(lib().perflibs_b200_tune_cache_save(os.fsencode(path)), "tune_cache_save")


def tune_cache_load(path):
    _check(lib().perflibs_b200_tune_cache_load(os.fsencode(path)), "tune_cache_load")


def tune_cache_clear():
    _check(lib().perflibs_b200_tune_cache_clear(), "tune_cache_clear")


def tune_cache_size():
    return int(lib().perflibs_b200_tune_cache_size())


def debug_guard_violations():
    """Writes past device buffers' ends seen by the guard build (-1 in the
    regular build)."""
    return int(lib().perflibs_b200_debug_guard_violations())


def spmm_optimize(transA, transB, alpha_hint, A: SpMat, B: SpMat, beta_hint, Cm: SpMat):
    return lib().perflibs_spmm_optimize(transA, transB, alpha_hint, A.h, B.h, beta_hint, Cm.h)


def read_mtx(path):
    """Matrix Market coordinate file -> (m, n, row_ptr, col, vals), 0-based
    CSR ordered by (row, column), symmetric files expanded (host only)."""
    L = lib()
    m, n, nnz = C.c_int32(), C.c_int32(), C.c_int64()
    rp, ci, vv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    st = L.perflibs_b200_read_mtx(os.fsencode(path), C.byref(m), C.byref(n), C.byref(nnz),
                                  C.byref(rp), C.byref(ci), C.byref(vv))
    _check(st, "read_mtx")
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    try:
        k = nnz.value
        row_ptr = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_int32)), (m.value + 1,)).copy()
        col = np.ctypeslib.as_array(C.cast(ci, C.POINTER(C.c_int32)), (max(k, 1),))[:k].copy()
        vals = np.ctypeslib.as_array(C.cast(vv, C.POINTER(C.c_double)), (max(k, 1),))[:k].copy()
    finally:
        for ptr in (rp, ci, vv):
            libc.free(ptr)
    return m.value, n.value, row_ptr, col, vals


def spmm_exec(transA, transB, alpha, A: SpMat, B: SpMat, beta, Cm: SpMat):
    fn = lib().perflibs_spmm_exec_s if A.dtype == np.float32 else lib().perflibs_spmm_exec_d
    return fn(transA, transB, alpha, A.h, B.h, beta, Cm.h)
