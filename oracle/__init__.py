"""CPU oracle for the block-iLDL^T + SQMR solve path -- TEST INFRASTRUCTURE ONLY.

A plain-C restatement of culip's libs/la solve path (see oracle.h / oracle_*.c
for the reference file:line each function follows).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline / reference leg may import
this package, and only as the checker; the product (culip_b200) never does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

# the FP32 factor's FP64 2x2-pivot bound (ORC_PIVOT_FP64_DEFAULT)
PIVOT_FP64_DEFAULT = 1e-3

_lib = None

_i32p = ctypes.POINTER(ctypes.c_int)


class _OrcSym(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int), ("nnz", ctypes.c_int), ("value_bytes", ctypes.c_int), ("num_blocks", ctypes.c_int),
        ("bs", _i32p), ("row_block", _i32p),
        ("coarse_nnz", ctypes.c_int), ("fill_nnz", ctypes.c_int),
        ("cs_off", _i32p), ("cs_col", _i32p), ("blk_nnzA", _i32p),
        ("csc_off", _i32p), ("csc_blk", _i32p),
        ("num_levels", ctypes.c_int), ("unleveled_rows", ctypes.c_int),
        ("lvl_off", _i32p), ("lvl_rows", _i32p), ("row_level", _i32p),
        ("max_level_size", ctypes.c_int), ("max_level_blocks", ctypes.c_int),
        ("lb_count", ctypes.c_int),
        ("lb_off", _i32p), ("lb", _i32p), ("sb_off", _i32p), ("sb", _i32p),
        ("blk_row", _i32p), ("blk_col", _i32p), ("fmt", _i32p), ("max_nnz", _i32p),
        ("a_blk", _i32p), ("a_idx", _i32p),
    ]


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.orc_symbolic.restype = ctypes.POINTER(_OrcSym)
        L.orc_symbolic.argtypes = [ctypes.c_int, vp, vp, ctypes.c_int, vp, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.orc_sym_free.argtypes = [vp]
        for sfx, real in (("_d", ctypes.c_double), ("_s", ctypes.c_float)):
            f = getattr(L, "orc_factor" + sfx)
            f.restype = vp
            f.argtypes = [vp, vp, vp, ctypes.c_int, real, ctypes.c_int]
            ff = getattr(L, "orc_factor_forced" + sfx)
            ff.restype = vp
            ff.argtypes = [vp, vp, vp, ctypes.c_int, real, ctypes.c_int, vp, ctypes.c_double]
            getattr(L, "orc_fac_free" + sfx).argtypes = [vp]
            g = getattr(L, "orc_fac_export_size" + sfx)
            g.restype = ctypes.c_long
            g.argtypes = [vp]
            getattr(L, "orc_fac_export" + sfx).argtypes = [vp] * 9
            getattr(L, "orc_prec_apply" + sfx).argtypes = [vp, ctypes.c_int, vp, vp]
            getattr(L, "orc_prec_apply_jacobi" + sfx).argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp]
        L.orc_spmv_d.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, ctypes.c_double, ctypes.c_double]
        L.orc_sqmr_d.restype = ctypes.c_int
        L.orc_sqmr_d.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, vp, ctypes.c_double, ctypes.c_int, vp]
        L.orc_sqmr_jacobi_d.restype = ctypes.c_int
        L.orc_sqmr_jacobi_d.argtypes = [ctypes.c_int, vp, vp, vp, vp, ctypes.c_int, vp, vp, ctypes.c_double,
                                        ctypes.c_int, vp]
        L.orc_sqmr_ldu_d.restype = ctypes.c_int
        L.orc_sqmr_ldu_d.argtypes = [ctypes.c_int] + [vp] * 12 + [ctypes.c_double, ctypes.c_int, vp]
        L.orc_ldu_apply_d.argtypes = [ctypes.c_int] + [vp] * 7 + [ctypes.c_int, vp, vp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_get_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    """Threads for the loops that are independent per row / block row (SpMV,
    vector updates, level sweeps, D); results do not depend on it."""
    lib().orc_set_threads(int(n))
    return lib().orc_get_threads()


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _arr(ptr, n):
    if n <= 0:
        return np.zeros(0, dtype=np.int32)
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy()


class Sym:
    """Symbolic analysis (BlockiLDLt ctor + symbolic part of compute())."""

    def __init__(self, rowptr, colidx, block_starts, fill_level=0, fill_factor=1.0, dtype=np.float64):
        self.rowptr = np.ascontiguousarray(rowptr, dtype=np.int32)
        self.colidx = np.ascontiguousarray(colidx, dtype=np.int32)
        bs = np.ascontiguousarray(block_starts, dtype=np.int32)
        self.n = len(self.rowptr) - 1
        if bs[-1] == self.n:
            bs = bs[:-1]
        self.num_blocks = len(bs)
        self.dtype = np.dtype(dtype)
        vb = self.dtype.itemsize
        self._h = lib().orc_symbolic(self.n, _p(self.rowptr), _p(self.colidx), self.num_blocks, _p(bs),
                                     fill_level, float(fill_factor), vb)
        s = self._h.contents
        cm, cnz, nl = s.num_blocks, s.coarse_nnz, s.num_levels
        self.coarse_nnz, self.fill_nnz, self.num_levels = cnz, s.fill_nnz, nl
        self.bs = _arr(s.bs, cm + 1)
        self.cs_off = _arr(s.cs_off, cm + 1)
        self.cs_col = _arr(s.cs_col, cnz)
        self.blk_nnzA = _arr(s.blk_nnzA, cnz)
        self.csc_off = _arr(s.csc_off, cm + 1)
        self.csc_blk = _arr(s.csc_blk, cnz)
        self.lvl_off = _arr(s.lvl_off, nl + 1)
        self.lvl_rows = _arr(s.lvl_rows, cm)
        self.lb_off = _arr(s.lb_off, nl + 1)
        self.lb = _arr(s.lb, cnz)
        self.sb_off = _arr(s.sb_off, nl + 1)
        self.sb = _arr(s.sb, cnz)
        self.fmt = _arr(s.fmt, cnz)
        self.max_nnz = _arr(s.max_nnz, cnz)
        self.blk_row = _arr(s.blk_row, cnz)
        self.blk_col = _arr(s.blk_col, cnz)
        self.unleveled_rows = s.unleveled_rows

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None:
            _lib.orc_sym_free(ctypes.cast(h, ctypes.c_void_p))
            self._h = None

    def factor(self, vals, is_piv=None, pivot=1, threshold=0.0, literal=False, forced_grants=None,
               pivot_fp64=PIVOT_FP64_DEFAULT) -> "Fac":
        """forced_grants: per block (block-id order) the extra slots a block
        that outgrows its capacity receives, as another run decided them.
        pivot_fp64: a float factor inverts 2x2 pivots whose ratio
        |d11 d22 - d12^2| / (|d11 d22| + d12^2) is below it in FP64 (0: float
        throughout, the reference's arithmetic)."""
        return Fac(self, vals, is_piv, pivot, threshold, literal, forced_grants, pivot_fp64)


class Fac:
    """Numeric factor (BlockiLDLt::factorize) and its applies."""

    def __init__(self, sym: Sym, vals, is_piv, pivot, threshold, literal, forced_grants=None,
                 pivot_fp64=None):
        self.sym = sym
        self.sfx = "_d" if sym.dtype == np.float64 else "_s"
        self.vals = np.ascontiguousarray(vals, dtype=sym.dtype)
        ip = np.ones(sym.n, np.int32) if is_piv is None else np.ascontiguousarray(is_piv, dtype=np.int32)
        self._forced = None
        if forced_grants is not None:
            self._forced = np.ascontiguousarray(forced_grants, dtype=np.int32)
            assert len(self._forced) == sym.coarse_nnz
        piv64 = PIVOT_FP64_DEFAULT if pivot_fp64 is None else float(pivot_fp64)
        f = getattr(lib(), "orc_factor_forced" + self.sfx)
        self._h = f(ctypes.cast(sym._h, ctypes.c_void_p), _p(self.vals), _p(ip), int(pivot), float(threshold),
                    1 if literal else 0, None if self._forced is None else _p(self._forced), piv64)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            getattr(_lib, "orc_fac_free" + self.sfx)(h)
            self._h = None

    def export(self) -> dict:
        L = lib()
        s = self.sym
        tot = getattr(L, "orc_fac_export_size" + self.sfx)(self._h)
        cnz = s.coarse_nnz
        out = dict(blk_nnz=np.zeros(cnz, np.int32), blk_off=np.zeros(cnz + 1, np.int64),
                   idx=np.zeros(max(tot, 1), np.int32), val=np.zeros(max(tot, 1), s.dtype),
                   tri=np.zeros(3 * s.n, s.dtype), is_piv=np.zeros(s.n, np.int32), perm=np.zeros(s.n, np.int32),
                   got_extra=np.zeros(cnz, np.int32))
        getattr(L, "orc_fac_export" + self.sfx)(self._h, _p(out["blk_nnz"]), _p(out["blk_off"]), _p(out["idx"]),
                                                _p(out["val"]), _p(out["tri"]), _p(out["is_piv"]), _p(out["perm"]),
                                                _p(out["got_extra"]))
        out["idx"] = out["idx"][:tot]
        out["val"] = out["val"][:tot]
        return out

    def apply(self, stage: int, b, jacobi_sweeps: int = 0) -> np.ndarray:
        """solve_left (0) / middle (1) / right (2); jacobi_sweeps > 0 replaces the
        exact triangular solves by that many block-Jacobi sweeps (SOLVE_JACOBI)."""
        b = np.ascontiguousarray(b, dtype=self.sym.dtype)
        x = np.zeros_like(b)
        if jacobi_sweeps > 0:
            getattr(lib(), "orc_prec_apply_jacobi" + self.sfx)(self._h, int(stage), int(jacobi_sweeps), _p(b), _p(x))
        else:
            getattr(lib(), "orc_prec_apply" + self.sfx)(self._h, int(stage), _p(b), _p(x))
        return x


def spmv(rowptr, colidx, val, x, alpha=1.0, beta=0.0, y=None) -> np.ndarray:
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    colidx = np.ascontiguousarray(colidx, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    m = len(rowptr) - 1
    y = np.zeros(m) if y is None else np.array(y, dtype=np.float64, copy=True)
    lib().orc_spmv_d(m, _p(rowptr), _p(colidx), _p(val), _p(x), _p(y), float(alpha), float(beta))
    return y


def sqmr(rowptr, colidx, val, b, fac: Fac | None = None, tol=1e-8, max_it=1000, jacobi_sweeps=0):
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    colidx = np.ascontiguousarray(colidx, np.int32)
    val = np.ascontiguousarray(val, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    m = len(rowptr) - 1
    x = np.zeros(m)
    res = np.zeros(1)
    if jacobi_sweeps > 0:
        it = lib().orc_sqmr_jacobi_d(m, _p(rowptr), _p(colidx), _p(val), fac._h, int(jacobi_sweeps), _p(b), _p(x),
                                     float(tol), int(max_it), _p(res))
        return x, float(res[0]), int(it)
    it = lib().orc_sqmr_d(m, _p(rowptr), _p(colidx), _p(val), fac._h if fac is not None else None, _p(b), _p(x),
                          float(tol), int(max_it), _p(res))
    return x, float(res[0]), int(it)


def sqmr_ldu(rowptr, colidx, val, L_rowptr, L_colidx, L_val, tri, is_piv, perm, scale, b, tol, max_it):
    a = [np.ascontiguousarray(v, t) for v, t in ((rowptr, np.int32), (colidx, np.int32), (val, np.float64),
                                                  (L_rowptr, np.int32), (L_colidx, np.int32), (L_val, np.float64),
                                                  (tri, np.float64), (is_piv, np.int32), (perm, np.int32),
                                                  (scale, np.float64), (b, np.float64))]
    m = len(a[0]) - 1
    x = np.zeros(m)
    res = np.zeros(1)
    it = lib().orc_sqmr_ldu_d(m, *[_p(v) for v in a], _p(x), float(tol), int(max_it), _p(res))
    return x, float(res[0]), int(it)


def ldu_apply(L_rowptr, L_colidx, L_val, tri, is_piv, perm, scale, stage, b):
    """ImportLDUPreconditioner::solve_left / middle / right (stage 0 / 1 / 2),
    import_ldu_preconditioner.impl.cuh, with the restatement's ldu_apply."""
    a = [np.ascontiguousarray(v, t) for v, t in ((L_rowptr, np.int32), (L_colidx, np.int32), (L_val, np.float64),
                                                  (tri, np.float64), (is_piv, np.int32), (perm, np.int32),
                                                  (scale, np.float64))]
    n = len(a[0]) - 1
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(n)
    lib().orc_ldu_apply_d(n, *[_p(v) for v in a], int(stage), _p(b), _p(x))
    return x


def kkt_assemble(m, n, a_rowptr, a_colidx, a_val, x=None, s=None, d=None, delta=1e-8, gamma=1e-8):
    """K = [[diag(d) + delta I, A'], [A, -gamma I]] with d = s / x (or given)
    as full symmetric CSR with sorted columns and an explicit diagonal (numpy
    restatement of the augmented system whose product AugmentedMatrixSPMV<T>
    computes, libs/la/spmv.cuh:104-149, with the dual shift on every row).
    Returns (rowptr, colidx, val)."""
    a_rowptr = np.asarray(a_rowptr, np.int64)
    a_colidx = np.asarray(a_colidx, np.int64)
    a_val = np.asarray(a_val, np.float64)
    dd = np.asarray(d, np.float64) if d is not None else np.asarray(s, np.float64) / np.asarray(x, np.float64)
    arow = np.repeat(np.arange(m), np.diff(a_rowptr))
    rows = np.concatenate([np.arange(n), a_colidx, n + arow, n + np.arange(m)])
    cols = np.concatenate([np.arange(n), n + arow, a_colidx, n + np.arange(m)])
    vals = np.concatenate([dd + delta, a_val, a_val, np.full(m, -gamma)])
    order = np.lexsort((cols, rows))
    rowptr = np.zeros(n + m + 1, np.int64)
    np.add.at(rowptr, rows + 1, 1)
    return np.cumsum(rowptr).astype(np.int32), cols[order].astype(np.int32), vals[order]


def permute_scale(rowptr, colidx, val, row_perm, col_perm=None, row_scale=None, col_scale=None,
                  scale_before_match=False, perm_is_old_to_new=True):
    """B = diag(1/r) P_r A P_c' diag(1/c) as sorted CSR (numpy restatement of
    T_matrix_permute_scale, libs/la/sparse_la.impl.cuh:599-657):
      * k_inv_perm (:586-595) inverts each given map when it is new -> old;
      * k_transform_coo (:552-582) maps every triplet (r, c, a) to
        (p_r[r], p_c[c], a / s), s = row_scale[r] * col_scale[c] when
        scale_before_match, else row_scale[p_r[r]] * col_scale[p_c[c]];
        without scales the reference divides by 1 (a value is unchanged);
      * T_coo2csr (:939-975) sorts the triplets by (row, column) (ties,
        i.e. duplicate entries, are kept in input order here).
    Returns (rowptr, colidx, val) of B; val keeps the input dtype."""
    rowptr = np.asarray(rowptr, np.int64)
    colidx = np.asarray(colidx, np.int64)
    val = np.asarray(val)
    n = len(rowptr) - 1

    def fwd(p):
        p = np.asarray(p, np.int64)
        if perm_is_old_to_new:
            return p
        inv = np.empty(n, np.int64)
        inv[p] = np.arange(n)
        return inv

    pr = fwd(row_perm)
    pc = pr if col_perm is None else fwd(col_perm)
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    new_r, new_c = pr[rows], pc[colidx]
    if row_scale is None:
        v = val.copy()
    else:
        rs = np.asarray(row_scale, val.dtype)
        cs = np.asarray(col_scale, val.dtype)
        sc = rs[rows] * cs[colidx] if scale_before_match else rs[new_r] * cs[new_c]
        v = val / sc
    order = np.lexsort((np.arange(len(val)), new_c, new_r))
    b_rowptr = np.zeros(n + 1, np.int32)
    np.add.at(b_rowptr, new_r + 1, 1)
    return np.cumsum(b_rowptr).astype(np.int32), new_c[order].astype(np.int32), v[order]


def kkt_operator(kind, rowptr, colidx, val, n, d, x, delta=0.0, ix=None, alpha=1.0, beta=0.0, y=None):
    """AugmentedMatrixSPMV<T>::multiply (kind 0) / NormalMatrixSPMV<T>::multiply
    (kind 1), libs/la/spmv.impl.cuh:214-269 and 364-427, in FP64 with numpy,
    for the operators those classes document (spmv.cuh:70-74, 103-107):
      kind 0: y = alpha [D x1 + A' x2 ; A x1 + (delta I)(ix) x2] + beta y
      kind 1: y = alpha (A D^-1 A' x + (delta I)(ix) x) + beta y
    Where the reference's code departs from them, this follows the documented
    operator: A' x2, not A' x1, in the augmented product (spmv.impl.cuh:416-420),
    and the shift at row ix[i] multiplies x[ix[i]] (k_add_app,
    helper_kernels.impl.cuh:361-374, multiplies x[i])."""
    import scipy.sparse as sp

    rowptr = np.asarray(rowptr)
    m = len(rowptr) - 1
    A = sp.csr_matrix((np.asarray(val, np.float64), np.asarray(colidx), rowptr), shape=(m, n))
    d = np.asarray(d, np.float64)
    x = np.asarray(x, np.float64)
    shift = np.zeros(m)
    if ix is not None:
        shift[np.asarray(ix)] = delta
    if kind == 0:
        x1, x2 = x[:n], x[n:]
        v = np.concatenate([d * x1 + A.T @ x2, A @ x1 + shift * x2])
    else:
        v = A @ ((A.T @ x) / d) + shift * x
    if beta == 0.0 or y is None:
        return alpha * v
    return alpha * v + beta * np.asarray(y, np.float64)
