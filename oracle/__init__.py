"""CPU oracle for the sparse x dense execute path — TEST INFRASTRUCTURE ONLY.

Two checkers live here:

* ``port``: ctypes bindings to ``_build/liboracle.so``, the plain-C
  restatement of the reference algorithms in ``plsparse_oracle.c`` (each
  routine cites the reference file:line it follows).
* ``ref``: ctypes bindings to ``_ref/libplsparse_ref.so``, the reference
  library compiled from its own sources by ``Makefile`` (target ``ref``),
  plus the hooks in ``ref_hooks.cpp``. Present only where that library was
  built.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package. The B200 library never does.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# PLSPARSE_ORACLE_LIB selects another build of the restatement (the
# sanitized one, for instance).
PORT_SO = os.environ.get("PLSPARSE_ORACLE_LIB") or os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libplsparse_ref.so")

_port = None
_ref = None


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def port():
    global _port
    if _port is None:
        if not os.path.exists(PORT_SO):
            raise RuntimeError(f"oracle port not built: {PORT_SO} (run `make -C oracle port`)")
        _port = C.CDLL(PORT_SO)
        L = _port
        vp, i32, i64, d, f = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_float
        L.orc_csr_spmv_d.argtypes = [i32, vp, vp, vp, vp, vp, d, d, C.c_int]
        L.orc_csr_spmv_s.argtypes = [i32, vp, vp, vp, vp, vp, f, f, C.c_int]
        L.orc_csr_spmv_trans_d.argtypes = [i32, i32, vp, vp, vp, vp, vp, d, d]
        L.orc_csr_absdot_d.argtypes = [i32, vp, vp, vp, vp, vp]
        L.orc_scs_sizes.argtypes = [i32, vp, i32, i32, vp]
        L.orc_scs_build_d.argtypes = [i32, i32, vp, vp, vp, i32, i32] + [vp] * 8
        L.orc_scs_spmv_d.argtypes = [i64, i32, vp, vp, vp, vp, vp, vp, vp, vp, d, d]
        L.orc_scs_beta.argtypes = [i64, i32, vp, vp, i32, i64]
        L.orc_scs_beta.restype = d
        L.orc_bsr_spmv_d.argtypes = [i32, i32, i32, vp, vp, vp, vp, vp, d, d]
        L.orc_bsr2csr_d.argtypes = [i32, i32, i32, vp, vp, vp, vp, vp, vp]
        L.orc_bsr2csr_d.restype = i64
        L.orc_csr2bsr_d.argtypes = [i32, i32, i32, i32, vp, vp, vp, vp, vp, vp]
        L.orc_csr2bsr_d.restype = i64
        L.orc_csr_spmm_d.argtypes = [i32, vp, vp, vp, vp, i64, vp, i64, i32, d, d]
        L.orc_csr_spmm_s.argtypes = [i32, vp, vp, vp, vp, i64, vp, i64, i32, f, f]
        L.orc_csr_inf_norm_d.argtypes = [i32, vp, vp]
        L.orc_csr_inf_norm_d.restype = d
        L.orc_coo2csr_d.argtypes = [i32, i32, i64, vp, vp, vp, vp, vp, vp]
        L.orc_csc2csr_d.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp]
    return _port


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise RuntimeError(f"reference oracle not built: {REF_SO}")
        _ref = C.CDLL(REF_SO)
        L = _ref
        vp, i32, i64, d, f = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_float
        L.perflibs_spmat_create_csr_d.argtypes = [vp, i32, i32, vp, vp, vp, i32]
        L.perflibs_spmat_create_csr_s.argtypes = [vp, i32, i32, vp, vp, vp, i32]
        L.perflibs_spmat_create_bsr_d.argtypes = [vp, C.c_int, i32, i32, i32, vp, vp, vp, i32]
        L.perflibs_spmat_create_coo_d.argtypes = [vp, i32, i32, i32, vp, vp, vp, i32]
        L.perflibs_spmat_create_csc_d.argtypes = [vp, i32, i32, vp, vp, vp, i32]
        L.perflibs_spmat_create_dense_d.argtypes = [vp, C.c_int, i32, i32, i32, vp, i32]
        L.perflibs_spmat_create_dense_s.argtypes = [vp, C.c_int, i32, i32, i32, vp, i32]
        L.perflibs_spmat_create_null.argtypes = [i32, i32]
        L.perflibs_spmat_create_null.restype = vp
        L.perflibs_spmat_hint.argtypes = [vp, C.c_int, C.c_int]
        L.perflibs_spmv_optimize.argtypes = [vp]
        L.perflibs_spmm_optimize.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, C.c_int, vp]
        L.perflibs_spmv_exec_d.argtypes = [C.c_int, d, vp, vp, d, vp]
        L.perflibs_spmv_exec_s.argtypes = [C.c_int, f, vp, vp, f, vp]
        L.perflibs_spmm_exec_d.argtypes = [C.c_int, C.c_int, d, vp, vp, d, vp]
        L.perflibs_spmm_exec_s.argtypes = [C.c_int, C.c_int, f, vp, vp, f, vp]
        L.perflibs_spmat_export_dense_d.argtypes = [vp, C.c_int, vp, vp, vp]
        L.perflibs_spmat_export_dense_s.argtypes = [vp, C.c_int, vp, vp, vp]
        L.perflibs_spmat_export_csr_d.argtypes = [vp, i32, vp, vp, vp, vp, vp]
        L.perflibs_spnorm_exec_d.argtypes = [vp, C.c_int, vp]
        L.perflibs_spmat_destroy.argtypes = [vp]
        L.ref_scs_build_d.argtypes = [i32, i32, vp, vp, vp, i32, i32, i32]
        L.ref_scs_build_d.restype = vp
        L.ref_scs_info.argtypes = [vp, vp]
        L.ref_scs_beta.argtypes = [vp, i32]
        L.ref_scs_beta.restype = d
        L.ref_scs_arrays.argtypes = [vp] * 8
        L.ref_scs_spmv_d.argtypes = [vp, vp, vp, d, d]
        L.ref_scs_free.argtypes = [vp]
        L.ref_set_C_sigma_d.argtypes = [vp, C.c_int, C.c_int]
        L.ref_set_time_limit_d.argtypes = [vp, d]
        L.ref_format_d.argtypes = [vp, vp, vp]
        L.free_ptr = C.CDLL(None).free
        L.free_ptr.argtypes = [vp]
    return _ref


# ----------------------------------------------------------------- port API


def csr_spmv(row_ptr, col, vals, x, y=None, alpha=1.0, beta=0.0, mode=1):
    """y = alpha*A*x + beta*y by the restated reference CSR kernel."""
    L = port()
    m = len(row_ptr) - 1
    if vals.dtype == np.float32:
        y = np.zeros(m, np.float32) if y is None else np.array(y, np.float32)
        L.orc_csr_spmv_s(m, _p(row_ptr), _p(col), _p(vals), _p(x), _p(y), alpha, beta, mode)
    else:
        y = np.zeros(m) if y is None else np.array(y, np.float64)
        L.orc_csr_spmv_d(m, _p(row_ptr), _p(col), _p(vals), _p(x), _p(y), alpha, beta, mode)
    return y


def csr_spmv_trans(row_ptr, col, vals, n, x, y=None, alpha=1.0, beta=0.0):
    L = port()
    m = len(row_ptr) - 1
    y = np.zeros(n) if y is None else np.array(y, np.float64)
    L.orc_csr_spmv_trans_d(m, n, _p(row_ptr), _p(col), _p(vals), _p(x), _p(y), alpha, beta)
    return y


def csr_absdot(row_ptr, col, vals, x):
    L = port()
    m = len(row_ptr) - 1
    out = np.zeros(m)
    L.orc_csr_absdot_d(m, _p(row_ptr), _p(col), _p(np.ascontiguousarray(vals, np.float64)),
                       _p(np.ascontiguousarray(x, np.float64)), _p(out))
    return out


def scs_build(row_ptr, col, vals, n, C, sigma):
    """Restated csr2scs + gen_data_vectors. Returns a dict of numpy arrays."""
    L = port()
    m = len(row_ptr) - 1
    sz = np.zeros(2, np.int64)
    L.orc_scs_sizes(m, _p(row_ptr), C, sigma, _p(sz))
    nC, size = int(sz[0]), int(sz[1])
    cs = np.zeros(max(nC, 1), np.int64)
    cl = np.zeros(max(nC, 1), np.int64)
    cm = np.zeros(max(nC, 1), np.int64)
    p2i = np.zeros(max(nC * C, 1), np.int64)
    i2p = np.zeros(max(nC * C, 1), np.int64)
    ov = np.zeros(max(size, 1))
    oo = np.zeros(max(size, 1), np.int64)
    info = np.zeros(3, np.int64)
    L.orc_scs_build_d(m, n, _p(row_ptr), _p(col), _p(np.ascontiguousarray(vals, np.float64)),
                      C, sigma, _p(cs), _p(cl), _p(cm), _p(p2i), _p(i2p), _p(ov), _p(oo), _p(info))
    return dict(nC=nC, C=C, sigma=sigma, size=size, cs=cs[:nC], cl=cl[:nC], col_min=cm[:nC],
                permd2in=p2i[: nC * C], in2permd=i2p[: nC * C], vals=ov[:size], offsets=oo[:size],
                col_bytes=int(info[0]), n_full_chunks=int(info[1]), ntidyup=int(info[2]))


def scs_spmv(s, x, y=None, alpha=1.0, beta=0.0):
    L = port()
    m = int((s["permd2in"] >= 0).sum())
    y = np.zeros(m) if y is None else np.array(y, np.float64)
    L.orc_scs_spmv_d(s["nC"], s["C"], _p(s["cs"]), _p(s["cl"]), _p(s["col_min"]),
                     _p(s["permd2in"]), _p(s["vals"]), _p(s["offsets"]), _p(x), _p(y), alpha, beta)
    return y


def scs_beta(s, nnz):
    L = port()
    return L.orc_scs_beta(s["nC"], s["C"], _p(s["cs"]), _p(s["cl"]), s["ntidyup"], nnz)


def bsr_spmv(row_ptr, col, vals, bs, layout, x, y=None, alpha=1.0, beta=0.0):
    L = port()
    nrowsb = len(row_ptr) - 1
    y = np.zeros(nrowsb * bs) if y is None else np.array(y, np.float64)
    L.orc_bsr_spmv_d(nrowsb, bs, layout, _p(row_ptr), _p(col), _p(vals), _p(x), _p(y), alpha, beta)
    return y


def bsr2csr(row_ptr, col, vals, bs, layout):
    L = port()
    nrowsb = len(row_ptr) - 1
    nnz = L.orc_bsr2csr_d(nrowsb, bs, layout, _p(row_ptr), _p(col), _p(vals), None, None, None)
    rp = np.zeros(nrowsb * bs + 1, np.int32)
    c = np.zeros(max(nnz, 1), np.int32)
    v = np.zeros(max(nnz, 1))
    L.orc_bsr2csr_d(nrowsb, bs, layout, _p(row_ptr), _p(col), _p(vals), _p(rp), _p(c), _p(v))
    return rp, c[:nnz], v[:nnz]


def csr2bsr(row_ptr, col, vals, m, n, bs, layout):
    L = port()
    nnzb = L.orc_csr2bsr_d(m, n, bs, layout, _p(row_ptr), _p(col), _p(vals), None, None, None)
    rp = np.zeros(m // bs + 1, np.int32)
    c = np.zeros(max(nnzb, 1), np.int32)
    v = np.zeros(max(nnzb * bs * bs, 1))
    L.orc_csr2bsr_d(m, n, bs, layout, _p(row_ptr), _p(col), _p(vals), _p(rp), _p(c), _p(v))
    return rp, c[:nnzb], v[: nnzb * bs * bs]


def csr_spmm(row_ptr, col, vals, B, k, Cmat=None, alpha=1.0, beta=0.0):
    """C = alpha*A*B + beta*C, B and C row-major (m x k)."""
    L = port()
    m = len(row_ptr) - 1
    if vals.dtype == np.float32:
        Cm = np.zeros((m, k), np.float32) if Cmat is None else np.array(Cmat, np.float32)
        if beta == 0:
            Cm[:] = 0
        L.orc_csr_spmm_s(m, _p(row_ptr), _p(col), _p(vals), _p(B), B.shape[1], _p(Cm), k, k, alpha, beta)
    else:
        Cm = np.zeros((m, k)) if Cmat is None else np.array(Cmat, np.float64)
        if beta == 0:
            Cm[:] = 0
        L.orc_csr_spmm_d(m, _p(row_ptr), _p(col), _p(vals), _p(B), B.shape[1], _p(Cm), k, k, alpha, beta)
    return Cm


def csr_inf_norm(row_ptr, vals):
    return port().orc_csr_inf_norm_d(len(row_ptr) - 1, _p(row_ptr), _p(vals))


def coo2csr(m, n, row, col, vals):
    """0-based COO -> CSR by (row, column), duplicates kept in input order."""
    row = np.ascontiguousarray(row, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    vals = np.ascontiguousarray(vals, np.float64)
    nnz = len(vals)
    rp = np.zeros(m + 1, np.int32)
    c = np.zeros(max(nnz, 1), np.int32)
    v = np.zeros(max(nnz, 1))
    port().orc_coo2csr_d(m, n, nnz, _p(row), _p(col), _p(vals), _p(rp), _p(c), _p(v))
    return rp, c[:nnz], v[:nnz]


def csc2csr(m, n, row_indx, col_ptr, vals):
    """CSC -> CSR with ascending columns per row (keeps col_ptr[0]'s base)."""
    row_indx = np.ascontiguousarray(row_indx, np.int32)
    col_ptr = np.ascontiguousarray(col_ptr, np.int32)
    vals = np.ascontiguousarray(vals, np.float64)
    nnz = int(col_ptr[n] - col_ptr[0])
    rp = np.zeros(m + 1, np.int32)
    c = np.zeros(max(nnz, 1), np.int32)
    v = np.zeros(max(nnz, 1))
    port().orc_csc2csr_d(m, n, _p(row_indx), _p(col_ptr), _p(vals), _p(rp), _p(c), _p(v))
    return rp, c[:nnz], v[:nnz]


# ------------------------------------------------------------ reference API


def ref_scs_build(row_ptr, col, vals, n, C, sigma, nthreads=1):
    """The reference's own csr2scs + gen_data_vectors, decoded to numpy."""
    L = ref()
    m = len(row_ptr) - 1
    h = L.ref_scs_build_d(m, n, _p(row_ptr), _p(col), _p(vals), C, sigma, nthreads)
    info = np.zeros(7, np.int64)
    L.ref_scs_info(h, _p(info))
    nC, Cc, sg, nb, nfull, ntidy, size = (int(v) for v in info)
    cs = np.zeros(max(nC, 1), np.int64)
    cl = np.zeros(max(nC, 1), np.int64)
    cm = np.zeros(max(nC, 1), np.int64)
    p2i = np.zeros(max(nC * Cc, 1), np.int64)
    i2p = np.zeros(max(nC * Cc, 1), np.int64)
    v = np.zeros(max(size, 1))
    raw = np.zeros(max(size * nb, 1), np.uint8)
    L.ref_scs_arrays(h, _p(cs), _p(cl), _p(cm), _p(p2i), _p(i2p), _p(v), _p(raw))
    beta = L.ref_scs_beta(h, int(row_ptr[-1] - row_ptr[0]))
    L.ref_scs_free(h)
    odt = {1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}[nb]
    offs = raw[: size * nb].view(odt).astype(np.int64)
    return dict(nC=nC, C=Cc, sigma=sg, size=size, cs=cs[:nC], cl=cl[:nC], col_min=cm[:nC],
                permd2in=p2i[: nC * Cc], in2permd=i2p[: nC * Cc], vals=v[:size], offsets=offs,
                col_bytes=nb, n_full_chunks=nfull, ntidyup=ntidy, beta=beta)


class RefMatrix:
    """A reference-library handle (CPU), used as the timed CPU baseline and
    as the end-to-end oracle for API-level parity tests."""

    def __init__(self, handle):
        self.h = handle

    @staticmethod
    def csr(m, n, row_ptr, col, vals):
        L = ref()
        h = C.c_void_p()
        fn = L.perflibs_spmat_create_csr_s if vals.dtype == np.float32 else L.perflibs_spmat_create_csr_d
        st = fn(C.byref(h), m, n, _p(row_ptr), _p(col), _p(vals), 0)
        if st != 0:
            raise RuntimeError(f"reference create_csr failed: {st}")
        return RefMatrix(h)

    @staticmethod
    def coo(m, n, row, col, vals):
        L = ref()
        h = C.c_void_p()
        row = np.ascontiguousarray(row, np.int32)
        col = np.ascontiguousarray(col, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        st = L.perflibs_spmat_create_coo_d(C.byref(h), m, n, len(vals), _p(row), _p(col), _p(vals), 0)
        if st != 0:
            raise RuntimeError(f"reference create_coo failed: {st}")
        return RefMatrix(h)

    @staticmethod
    def csc(m, n, row_indx, col_ptr, vals):
        L = ref()
        h = C.c_void_p()
        row_indx = np.ascontiguousarray(row_indx, np.int32)
        col_ptr = np.ascontiguousarray(col_ptr, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        st = L.perflibs_spmat_create_csc_d(C.byref(h), m, n, _p(row_indx), _p(col_ptr), _p(vals), 0)
        if st != 0:
            raise RuntimeError(f"reference create_csc failed: {st}")
        return RefMatrix(h)

    @staticmethod
    def bsr(layout, m, n, bs, row_ptr, col, vals):
        L = ref()
        h = C.c_void_p()
        row_ptr = np.ascontiguousarray(row_ptr, np.int32)
        col = np.ascontiguousarray(col, np.int32)
        vals = np.ascontiguousarray(vals, np.float64)
        st = L.perflibs_spmat_create_bsr_d(C.byref(h), layout, m, n, bs, _p(row_ptr), _p(col), _p(vals), 0)
        if st != 0:
            raise RuntimeError(f"reference create_bsr failed: {st}")
        return RefMatrix(h)

    @staticmethod
    def dense(M: np.ndarray):
        """A row-major dense handle (the reference copies the values)."""
        L = ref()
        h = C.c_void_p()
        M = np.ascontiguousarray(M, np.float64)
        rows, cols = M.shape
        st = L.perflibs_spmat_create_dense_d(C.byref(h), 91, rows, cols, cols, _p(M), 0)
        if st != 0:
            raise RuntimeError(f"reference create_dense failed: {st}")
        return RefMatrix(h)

    def export_dense(self):
        """Row-major values of a dense handle (the reference's export_dense)."""
        L = ref()
        rows, cols = C.c_int32(), C.c_int32()
        vv = C.c_void_p()
        st = L.perflibs_spmat_export_dense_d(self.h, 91, C.byref(rows), C.byref(cols), C.byref(vv))
        if st != 0:
            raise RuntimeError(f"reference export_dense failed: {st}")
        cnt = rows.value * cols.value
        out = np.ctypeslib.as_array(C.cast(vv, C.POINTER(C.c_double)), (max(cnt, 1),))[:cnt].copy()
        L.free_ptr(vv)
        return out.reshape(rows.value, cols.value)

    def spmm(self, m, B, alpha=1.0, beta=0.0, C0=None):
        """C = alpha * A * B + beta * C0 through the reference's own
        perflibs_spmm_exec_d (NOTRANS, NOTRANS): B a dense row-major handle,
        C a null handle when C0 is None (the reference materialises it) or a
        dense copy of C0. Returns C as an m x k FP64 array."""
        L = ref()
        Bh = RefMatrix.dense(B)
        k = B.shape[1]
        if C0 is None:
            Ch = RefMatrix(C.c_void_p(L.perflibs_spmat_create_null(m, k)))
        else:
            Ch = RefMatrix.dense(C0)
        st = L.perflibs_spmm_exec_d(300, 300, alpha, self.h, Bh.h, beta, Ch.h)
        if st != 0:
            raise RuntimeError(f"reference spmm_exec failed: {st}")
        out = Ch.export_dense()
        Bh.destroy()
        Ch.destroy()
        return out

    def export_csr(self, m, index_base=0):
        """The reference's own export (it converts the handle to CSR first)."""
        L = ref()
        rows, cols = C.c_int32(), C.c_int32()
        rp, ci, vv = C.c_void_p(), C.c_void_p(), C.c_void_p()
        st = L.perflibs_spmat_export_csr_d(self.h, index_base, C.byref(rows), C.byref(cols),
                                           C.byref(rp), C.byref(ci), C.byref(vv))
        if st != 0:
            raise RuntimeError(f"reference export_csr failed: {st}")
        r = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_int32)), (rows.value + 1,)).copy()
        nnz = int(r[-1] - r[0])
        c = np.ctypeslib.as_array(C.cast(ci, C.POINTER(C.c_int32)), (max(nnz, 1),))[:nnz].copy()
        v = np.ctypeslib.as_array(C.cast(vv, C.POINTER(C.c_double)), (max(nnz, 1),))[:nnz].copy()
        for ptr in (rp, ci, vv):
            L.free_ptr(ptr)
        return r, c, v

    def hint(self, hint, value):
        return ref().perflibs_spmat_hint(self.h, hint, value)

    def optimize(self):
        return ref().perflibs_spmv_optimize(self.h)

    def spmv(self, x, y, alpha=1.0, beta=0.0, trans=300):
        L = ref()
        if x.dtype == np.float32:
            return L.perflibs_spmv_exec_s(trans, alpha, self.h, _p(x), beta, _p(y))
        return L.perflibs_spmv_exec_d(trans, alpha, self.h, _p(x), beta, _p(y))

    def format(self):
        c, s = C.c_int(), C.c_int()
        f = ref().ref_format_d(self.h, C.byref(c), C.byref(s))
        return f, c.value, s.value

    def destroy(self):
        if self.h:
            ref().perflibs_spmat_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass
