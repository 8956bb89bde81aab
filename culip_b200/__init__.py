"""culip_b200: B200-native block-iLDL^T + SQMR solve path for KKT systems.

Python mirror of the reference's class API over the C ABI (include/culipx.h):

  BlockiLDLt      libs/la/preconditioner/block_ildlt.cuh:188-401
  CSRMatrixSPMV   libs/la/spmv.cuh:19-66
  SQMR            libs/la/iterative_solvers/sqmr.cuh:29-79

plus the lower-level objects they are built from (Handle, Pattern, Factor,
CsrOperator) and the seeded KKT generator.  Device vectors are torch CUDA
tensors (PyTorch is used only for device memory and streams); all compute
runs in libculipx.so's sm_100a kernels.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi as capi
from ._capi import (F32, F64, FMT_CSR, FMT_SELL, LEFT, MIDDLE, PIV_BK, PIV_ROOK, PIV_STATIC, RIGHT,  # noqa: F401
                    SOLVE_BLOCK, SOLVE_JACOBI, SOLVE_SCALAR, SOLVE_STRIPE, CulipxError, KktSpec)

__all__ = ["Handle", "Pattern", "Factor", "CsrOperator", "PermutePlan", "BlockiLDLt", "CSRMatrixSPMV", "SQMR", "kkt_generate",
           "kkt_blocking", "normal_vector", "CulipxError", "KKT_CONFIGS"]

# The benchmark systems: K = [[H + delta I, A'], [A, -gamma I]] with H diagonal, log-uniform in
# [hmin, hmax], and nnz_per_col N(0,1) entries per column of A (culipx_kkt_generate)
KKT_CONFIGS = {
    "small": dict(n=2000, m=1000, nnz_per_col=4, band_half=0, hmin=1e-2, hmax=1e2, block=4),
    "scale": dict(n=200000, m=100000, nnz_per_col=6, band_half=32, hmin=1e-6, hmax=1e6, block=32),
    "mixed": dict(n=1000000, m=500000, nnz_per_col=6, band_half=32, hmin=1e-6, hmax=1e6, block=32),
}
SEED = 20260101


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _dptr(t) -> ctypes.c_void_p:
    """Device pointer of a torch CUDA tensor (or None)."""
    if t is None:
        return None
    if not getattr(t, "is_cuda", False):
        raise TypeError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


def _release(obj, destroy: str):
    """Destroys obj's C handle once; a no-op while the interpreter shuts down
    (module globals may already be gone then)."""
    h = getattr(obj, "_h", None)
    if h is None or not h.value:
        return
    try:
        lib = capi._lib
        if lib is not None:
            getattr(lib, destroy)(h)
    except Exception:
        pass
    obj._h = None


def kkt_generate(n, m, nnz_per_col, band_half, hmin, hmax, delta=1e-8, gamma=1e-8, seed=SEED):
    """Seeded KKT system as full symmetric CSR (rowptr, colidx, val) numpy arrays."""
    spec = KktSpec(n, m, nnz_per_col, band_half, hmin, hmax, delta, gamma, seed)
    nnz = ctypes.c_longlong()
    capi.call("culipx_kkt_nnz", ctypes.byref(spec), ctypes.byref(nnz))
    rowptr = np.zeros(n + m + 1, np.int32)
    colidx = np.zeros(nnz.value, np.int32)
    val = np.zeros(nnz.value, np.float64)
    capi.call("culipx_kkt_generate", ctypes.byref(spec), _p(rowptr), _p(colidx), _p(val))
    return rowptr, colidx, val


def kkt_blocking(n, m, block) -> np.ndarray:
    """block_starts with num_blocks + 1 entries (last = n + m)."""
    nb = ctypes.c_int()
    capi.call("culipx_kkt_blocking", n, m, block, None, 0, ctypes.byref(nb))
    bs = np.zeros(nb.value + 1, np.int32)
    capi.call("culipx_kkt_blocking", n, m, block, _p(bs), nb.value + 1, ctypes.byref(nb))
    return bs


def blocking_generate(rowptr, colidx, min_size=8, max_size=32) -> np.ndarray:
    """block_starts (num_blocks + 1 entries, last = n) for any symmetric
    pattern, from culipx_blocking_generate."""
    rp = np.ascontiguousarray(rowptr, np.int32)
    ci = np.ascontiguousarray(colidx, np.int32)
    n = len(rp) - 1
    nb = ctypes.c_int()
    capi.call("culipx_blocking_generate", n, _p(rp), _p(ci), int(min_size), int(max_size), None, 0, ctypes.byref(nb))
    bs = np.zeros(nb.value + 1, np.int32)
    capi.call("culipx_blocking_generate", n, _p(rp), _p(ci), int(min_size), int(max_size), _p(bs), nb.value + 1,
              ctypes.byref(nb))
    return bs


def normal_vector(seed, n) -> np.ndarray:
    out = np.zeros(n, np.float64)
    capi.call("culipx_normal_vector", seed, n, _p(out))
    return out


class Handle:
    """Device, stream and device-memory budget (the reference's gpu_handle_t)."""

    def __init__(self, device: int = 0, stream=None):
        import torch

        self.device = device
        if stream is None:
            stream = torch.cuda.current_stream(device)
        self.stream = stream
        h = ctypes.c_void_p()
        capi.call("culipx_handle_create", ctypes.byref(h), device, ctypes.c_void_p(stream.cuda_stream))
        self._h = h

    def set_stream(self, stream):
        self.stream = stream
        capi.call("culipx_handle_set_stream", self._h, ctypes.c_void_p(stream.cuda_stream))

    def set_memory_budget(self, nbytes: int):
        capi.call("culipx_handle_set_memory_budget", self._h, int(nbytes))

    def memory_used(self) -> int:
        v = ctypes.c_longlong()
        capi.call("culipx_handle_memory_used", self._h, ctypes.byref(v))
        return v.value

    def synchronize(self):
        capi.call("culipx_handle_synchronize", self._h)

    def launch_count(self, reset=False) -> int:
        v = ctypes.c_longlong()
        capi.call("culipx_handle_launch_count", self._h, ctypes.byref(v), 1 if reset else 0)
        return v.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            capi.load().culipx_handle_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Pattern:
    """Symbolic analysis of one sparsity pattern (BlockiLDLt ctor + symbolic part of compute())."""

    def __init__(self, handle: Handle, rowptr, colidx, block_starts, fill_level=0, fill_factor=1.0,
                 precision=F64, system_row_offsets=None):
        self.handle = handle
        self.rowptr = np.ascontiguousarray(rowptr, np.int32)
        self.colidx = np.ascontiguousarray(colidx, np.int32)
        self.n = len(self.rowptr) - 1
        bs = np.ascontiguousarray(block_starts, np.int32)
        if bs[-1] == self.n:
            bs = bs[:-1]
        self.num_blocks = len(bs)
        self.precision = precision
        p = ctypes.c_void_p()
        if system_row_offsets is None:
            capi.call("culipx_pattern_analyze", handle._h, self.n, _p(self.rowptr), _p(self.colidx), self.num_blocks,
                      _p(bs), int(fill_level), float(fill_factor), int(precision), ctypes.byref(p))
        else:
            so = np.ascontiguousarray(system_row_offsets, np.int32)
            capi.call("culipx_pattern_analyze_systems", handle._h, self.n, _p(self.rowptr), _p(self.colidx),
                      self.num_blocks, _p(bs), int(fill_level), float(fill_factor), int(precision), len(so) - 1,
                      _p(so), ctypes.byref(p))
        self._h = p

    def info(self) -> dict:
        v = np.zeros(16, np.int64)
        capi.call("culipx_pattern_info", self._h, _p(v))
        keys = ["n", "nnz", "num_blocks", "coarse_nnz", "fill_nnz", "num_levels", "num_sparse", "num_dense",
                "val_slots", "idx_slots", "max_level_blocks", "max_level_rows", "device_bytes", "precision"]
        return {k: int(v[i]) for i, k in enumerate(keys)}

    def export(self) -> dict:
        inf = self.info()
        cm, cnz, nl = inf["num_blocks"], inf["coarse_nnz"], inf["num_levels"]
        out = dict(coarse_off=np.zeros(cm + 1, np.int32), coarse_col=np.zeros(cnz, np.int32),
                   blk_nnzA=np.zeros(cnz, np.int32), lvl_off=np.zeros(nl + 1, np.int32),
                   lvl_rows=np.zeros(cm, np.int32), lb_off=np.zeros(nl + 1, np.int32), lb=np.zeros(cnz, np.int32),
                   sb_off=np.zeros(nl + 1, np.int32), sb=np.zeros(cnz, np.int32), fmt=np.zeros(cnz, np.int32),
                   max_nnz=np.zeros(cnz, np.int32))
        capi.call("culipx_pattern_export", self._h, *[_p(out[k]) for k in
                                                      ("coarse_off", "coarse_col", "blk_nnzA", "lvl_off", "lvl_rows",
                                                       "lb_off", "lb", "sb_off", "sb", "fmt", "max_nnz")])
        return out

    def __del__(self):
        try:
            _release(self, "culipx_pattern_destroy")
        except Exception:  # interpreter shutdown
            pass


class Factor:
    """Numeric block-iLDL^T factor of one pattern (BlockiLDLt::factorize + applies)."""

    def __init__(self, pattern: Pattern):
        self.pattern = pattern
        f = ctypes.c_void_p()
        capi.call("culipx_factor_create", pattern._h, ctypes.byref(f))
        self._h = f

    @property
    def dtype(self):
        import torch

        return torch.float64 if self.pattern.precision == F64 else torch.float32

    def compute(self, vals, is_piv=None, pivot=PIV_BK, threshold=0.0):
        """vals: torch CUDA tensor (pattern precision) or host numpy float64 array."""
        ip = None if is_piv is None else np.ascontiguousarray(is_piv, np.int32)
        if isinstance(vals, np.ndarray):
            v = np.ascontiguousarray(vals, np.float64)
            capi.call("culipx_factor_compute_host", self._h, _p(v), None if ip is None else _p(ip), int(pivot),
                      float(threshold))
        else:
            self._check_values(vals)
            capi.call("culipx_factor_compute", self._h, _dptr(vals), None if ip is None else _p(ip), int(pivot),
                      float(threshold))

    def _check_values(self, vals):
        """The C ABI takes raw pointers: refuse a values tensor whose type or
        length differs from the pattern's, which the kernels would misread."""
        if vals.dtype != self.dtype:
            raise TypeError(f"values must be {self.dtype} for this pattern's precision, got {vals.dtype}")
        nnz = int(self.pattern.rowptr[-1])
        if vals.numel() < nnz:
            raise ValueError(f"values hold {vals.numel()} entries, the pattern has {nnz}")

    def compute_graph(self, vals, pivot=PIV_BK, threshold=0.0):
        """compute() replayed from a CUDA graph captured on the first call
        for this tensor (vals: torch CUDA tensor, pattern precision)."""
        self._check_values(vals)
        capi.call("culipx_factor_compute_graph", self._h, _dptr(vals), int(pivot), float(threshold))

    def set_solve_algorithm(self, algorithm, sweeps=0):
        capi.call("culipx_factor_set_solve_algorithm", self._h, int(algorithm), int(sweeps))

    def set_pivot_fp64(self, bound):
        """FP32 factors: 2x2 pivots with |d11 d22 - d12^2| / (|d11 d22| + d12^2)
        below bound are inverted in FP64 (default 1e-3; 0 = the reference's
        FP32 arithmetic).  Used by the next compute."""
        capi.call("culipx_factor_set_pivot_fp64", self._h, float(bound))

    def stats(self):
        ms = ctypes.c_double()
        nl = ctypes.c_int()
        capi.call("culipx_factor_stats", self._h, ctypes.byref(ms), ctypes.byref(nl))
        return ms.value, nl.value

    def info(self) -> dict:
        """Sizes of the solve structures of the last computed factor."""
        out = np.zeros(8, dtype=np.int64)
        capi.call("culipx_factor_info", self._h, out.ctypes.data_as(ctypes.c_void_p))
        keys = ["u_nnz", "tiles", "tile_entries", "simple_rows", "blocks_2x2", "value_bytes", "granted_blocks"]
        return {k: int(v) for k, v in zip(keys, out)}

    def export(self) -> dict:
        tot = ctypes.c_longlong()
        capi.call("culipx_factor_export_size", self._h, ctypes.byref(tot))
        inf = self.pattern.info()
        cnz, n = inf["coarse_nnz"], inf["n"]
        vd = np.float64 if self.pattern.precision == F64 else np.float32
        out = dict(blk_nnz=np.zeros(cnz, np.int32), blk_off=np.zeros(cnz + 1, np.int64),
                   idx=np.zeros(max(tot.value, 1), np.int32), val=np.zeros(max(tot.value, 1), vd),
                   tri=np.zeros(3 * n, vd), is_piv=np.zeros(n, np.int32), perm=np.zeros(n, np.int32),
                   got_extra=np.zeros(cnz, np.int32))
        capi.call("culipx_factor_export", self._h, *[_p(out[k]) for k in
                                                     ("blk_nnz", "blk_off", "idx", "val", "tri", "is_piv", "perm",
                                                      "got_extra")])
        out["idx"] = out["idx"][: tot.value]
        out["val"] = out["val"][: tot.value]
        return out

    def apply(self, stage: int, b, x=None):
        import torch

        if x is None:
            x = torch.empty_like(b)
        capi.call("culipx_prec_apply", self._h, int(stage), _dptr(b), _dptr(x))
        return x

    def __del__(self):
        try:
            _release(self, "culipx_factor_destroy")
        except Exception:  # interpreter shutdown
            pass


class PermutePlan:
    """B = diag(1/r) P_r K P_c' diag(1/c), sorted (T_matrix_permute_scale /
    host_permute).  Built once per pattern from device rowptr/colidx and host
    permutations; apply() maps a device value array into B's order."""

    def __init__(self, handle: Handle, d_rowptr, d_colidx, row_perm, col_perm=None, perm_is_old_to_new=True):
        self.handle = handle
        self.n = int(d_rowptr.numel()) - 1
        self.nnz = int(d_colidx.numel())
        rp = np.ascontiguousarray(row_perm, np.int32)
        cp = None if col_perm is None else np.ascontiguousarray(col_perm, np.int32)
        h = ctypes.c_void_p()
        capi.call("culipx_permute_create", handle._h, self.n, self.nnz, _dptr(d_rowptr), _dptr(d_colidx),
                  rp.ctypes.data_as(ctypes.c_void_p), None if cp is None else cp.ctypes.data_as(ctypes.c_void_p),
                  int(bool(perm_is_old_to_new)), ctypes.byref(h))
        self._h = h

    def structure(self):
        """(rowptr, colidx) of B as host numpy int32 arrays."""
        rowptr = np.zeros(self.n + 1, np.int32)
        colidx = np.zeros(max(self.nnz, 1), np.int32)
        capi.call("culipx_permute_export", self._h, rowptr.ctypes.data_as(ctypes.c_void_p),
                  colidx.ctypes.data_as(ctypes.c_void_p))
        return rowptr, colidx[: self.nnz]

    def apply(self, d_val, d_out, row_scale=None, col_scale=None, scale_before_match=False):
        prec = F64 if d_val.dtype.itemsize == 8 else F32
        capi.call("culipx_permute_apply", self._h, prec, _dptr(d_val), _dptr(row_scale), _dptr(col_scale),
                  int(bool(scale_before_match)), _dptr(d_out))

    def __del__(self):
        try:
            _release(self, "culipx_permute_destroy")
        except Exception:  # interpreter shutdown
            pass


def sprank(m: int, n: int, rowptr, colidx):
    """Structural rank of an m x n CSR pattern (culipx_sprank, culip's
    sprank): (rank, row_match, col_match), INT_MAX marking unmatched."""
    rp = np.ascontiguousarray(rowptr, np.int32)
    ci = np.ascontiguousarray(colidx, np.int32)
    rmatch = np.zeros(max(m, 1), np.int32)
    cmatch = np.zeros(max(n, 1), np.int32)
    rank = ctypes.c_int()
    capi.call("culipx_sprank", int(m), int(n), _p(rp), _p(ci), _p(rmatch), _p(cmatch), ctypes.byref(rank))
    return rank.value, rmatch[:m], cmatch[:n]


def ordering_rcm(rowptr, colidx):
    """Reverse Cuthill-McKee ordering of a square CSR pattern
    (culipx_ordering_rcm): perm[new] = old."""
    rp = np.ascontiguousarray(rowptr, np.int32)
    ci = np.ascontiguousarray(colidx, np.int32)
    n = len(rp) - 1
    perm = np.zeros(max(n, 1), np.int32)
    capi.call("culipx_ordering_rcm", n, _p(rp), _p(ci), _p(perm))
    return perm[:n]


class KktAssembly:
    """K = [[diag(d) + delta I, A'], [A, -gamma I]] of an interior-point
    iteration, d = s / x (or given), as full symmetric CSR: the structure is
    planned once per pattern of A (m x n CSR, torch int32 CUDA tensors),
    assemble() writes one iteration's values on the device."""

    def __init__(self, handle: Handle, m: int, n: int, d_rowptr, d_colidx):
        self.handle = handle
        self.m, self.n = int(m), int(n)
        self._keep = (d_rowptr, d_colidx)
        h = ctypes.c_void_p()
        capi.call("culipx_kkt_assembly_create", handle._h, self.m, self.n, int(d_colidx.numel()), _dptr(d_rowptr),
                  _dptr(d_colidx), ctypes.byref(h))
        self._h = h
        N = ctypes.c_int()
        nnz = ctypes.c_longlong()
        capi.call("culipx_kkt_assembly_size", self._h, ctypes.byref(N), ctypes.byref(nnz))
        self.N, self.nnz = N.value, nnz.value

    def structure(self):
        """(rowptr, colidx) of K as host numpy int32 arrays."""
        rowptr = np.zeros(self.N + 1, np.int32)
        colidx = np.zeros(max(self.nnz, 1), np.int32)
        capi.call("culipx_kkt_assembly_export", self._h, _p(rowptr), _p(colidx))
        return rowptr, colidx[: self.nnz]

    def assemble(self, d_aval, d_kval, x=None, s=None, d=None, delta=1e-8, gamma=1e-8):
        """K's values into d_kval (float64 or float32 CUDA tensor of nnz
        entries) from A's values and the iterate (x, s) or the diagonal d."""
        prec = F64 if d_kval.dtype.itemsize == 8 else F32
        capi.call("culipx_kkt_assemble", self._h, _dptr(d_aval), _dptr(x), _dptr(s), _dptr(d), float(delta),
                  float(gamma), prec, _dptr(d_kval))
        return d_kval

    def __del__(self):
        try:
            _release(self, "culipx_kkt_assembly_destroy")
        except Exception:  # interpreter shutdown
            pass


class CsrOperator:
    """CSR operator over torch CUDA tensors (kept alive by this object)."""

    def __init__(self, handle: Handle, rowptr, colidx, val, ncols=None, explicit_transpose=False):
        self.handle = handle
        self.rowptr, self.colidx, self.val = rowptr, colidx, val
        self.m = rowptr.numel() - 1
        self.n = self.m if ncols is None else ncols
        import torch

        prec = F64 if val.dtype == torch.float64 else F32
        A = ctypes.c_void_p()
        capi.call("culipx_csr_create", handle._h, self.m, self.n, colidx.numel(), _dptr(rowptr), _dptr(colidx),
                  _dptr(val), prec, 1 if explicit_transpose else 0, ctypes.byref(A))
        self._h = A

    def spmv(self, x, y, alpha=1.0, beta=0.0, transpose=False):
        capi.call("culipx_spmv", self._h, _dptr(x), _dptr(y), float(alpha), float(beta), 1 if transpose else 0)
        return y

    def set_format(self, fmt):
        """FMT_CSR (the borrowed arrays) or FMT_SELL (a SELL-32 copy of
        structure and values, built now; refresh() after changing val)."""
        capi.call("culipx_csr_set_format", self._h, int(fmt))

    def refresh(self):
        capi.call("culipx_csr_refresh", self._h)

    def __del__(self):
        try:
            _release(self, "culipx_csr_destroy")
        except Exception:  # interpreter shutdown
            pass


def sqmr_solve(handle: Handle, A: CsrOperator, M: Factor | None, b, x, tol=1e-8, max_it=1000):
    """Returns (residual, iterations, status); status is OK or MAXIT."""
    res = ctypes.c_double()
    its = ctypes.c_int()
    st = capi.call("culipx_sqmr_solve", handle._h, A._h, M._h if M is not None else None, _dptr(b), _dptr(x),
                   float(tol), int(max_it), ctypes.byref(res), ctypes.byref(its), allow=(capi.OK, capi.MAXIT))
    return res.value, its.value, st


def union_systems(systems):
    """Block-diagonal union of independent systems, each (rowptr, colidx, val,
    block_starts) with block_starts ending at its n.  Returns (rowptr, colidx,
    val, block_starts, row_offsets) of the union."""
    rps, cis, vs, bss, offs = [], [], [], [], [0]
    nnz = 0
    for rp, ci, v, bs in systems:
        rp = np.asarray(rp, np.int64)
        n0 = offs[-1]
        rps.append(rp[:-1] + nnz)
        cis.append(np.asarray(ci, np.int64) + n0)
        vs.append(np.asarray(v))
        b = np.asarray(bs, np.int64)
        bss.append((b[:-1] if b[-1] == len(rp) - 1 else b) + n0)
        nnz += int(rp[-1])
        offs.append(n0 + len(rp) - 1)
    rowptr = np.concatenate(rps + [np.array([nnz])]).astype(np.int32)
    bs = np.concatenate(bss + [np.array([offs[-1]])]).astype(np.int32)
    return rowptr, np.concatenate(cis).astype(np.int32), np.concatenate(vs), bs, np.asarray(offs, np.int32)


class Batch:
    """Independent systems stored as consecutive row ranges of one union
    pattern, solved together by batch_sqmr_solve (one CTA per system)."""

    def __init__(self, pattern: Pattern, row_offsets):
        self.pattern = pattern
        self.row_offsets = np.ascontiguousarray(row_offsets, np.int32)
        self.num = len(self.row_offsets) - 1
        h = ctypes.c_void_p()
        capi.call("culipx_batch_create", pattern._h, self.num, _p(self.row_offsets), ctypes.byref(h))
        self._h = h

    def __del__(self):
        try:
            _release(self, "culipx_batch_destroy")
        except Exception:  # interpreter shutdown
            pass


def batch_sqmr_solve(batch: Batch, A: CsrOperator, M: Factor, b, x, tol=1e-8, max_it=1000):
    """Returns per-system (residual, iterations, status) numpy arrays."""
    res = np.zeros(batch.num)
    its = np.zeros(batch.num, np.int32)
    st = np.zeros(batch.num, np.int32)
    capi.call("culipx_batch_sqmr_solve", batch._h, A._h, M._h, _dptr(b), _dptr(x), float(tol), int(max_it), _p(res),
              _p(its), _p(st))
    return res, its, st


def batch_factor_solve_graph(batch: Batch, A: CsrOperator, M: Factor, vals, b, x, tol=1e-8, max_it=1000,
                             pivot=PIV_BK, threshold=0.0):
    """Factor the union (values `vals`, a CUDA tensor in M's precision) and
    solve all systems, as one CUDA-graph launch after the first call for the
    same buffers (culipx_batch_factor_solve_graph).  Returns per-system
    (residual, iterations, status) numpy arrays."""
    res = np.zeros(batch.num)
    its = np.zeros(batch.num, np.int32)
    st = np.zeros(batch.num, np.int32)
    capi.call("culipx_batch_factor_solve_graph", batch._h, A._h, M._h, _dptr(vals), int(pivot), float(threshold),
              _dptr(b), _dptr(x), float(tol), int(max_it), _p(res), _p(its), _p(st))
    return res, its, st


class Server:
    """Continuous-batching request server (culipx_server_*): patterns analysed
    once, requests (K's values + right-hand sides, host numpy) admitted by
    device memory into batched launches on several streams."""

    def __init__(self, device=0, memory_budget=0, slots=2, max_batch=256, tol=1e-8, max_it=1000):
        h = ctypes.c_void_p()
        capi.call("culipx_server_create", int(device), int(memory_budget), int(slots), int(max_batch), float(tol),
                  int(max_it), ctypes.byref(h))
        self._h = h
        self.patterns = []

    def add_pattern(self, rowptr, colidx, block_starts, precision=F64) -> int:
        rp = np.ascontiguousarray(rowptr, np.int32)
        ci = np.ascontiguousarray(colidx, np.int32)
        bs = np.ascontiguousarray(block_starts, np.int32)
        n = len(rp) - 1
        if bs[-1] == n:
            bs = bs[:-1]
        pid = ctypes.c_int()
        capi.call("culipx_server_add_pattern", self._h, n, _p(rp), _p(ci), len(bs), _p(bs), int(precision),
                  ctypes.byref(pid))
        self.patterns.append((n, len(ci)))
        return pid.value

    def submit(self, pid, vals, b) -> int:
        v = np.ascontiguousarray(vals, np.float64)
        b = np.asarray(b, np.float64)
        nrhs = 1 if b.ndim == 1 else b.shape[1]
        bb = np.ascontiguousarray(b.reshape(-1, nrhs).T if b.ndim == 2 else b)
        rid = ctypes.c_int()
        capi.call("culipx_server_submit", self._h, int(pid), _p(v), nrhs, _p(bb), ctypes.byref(rid))
        self._meta = getattr(self, "_meta", {})
        self._meta[rid.value] = (pid, nrhs)
        return rid.value

    def progress(self, wait=False) -> int:
        c = ctypes.c_int()
        capi.call("culipx_server_progress", self._h, 1 if wait else 0, ctypes.byref(c))
        return c.value

    def result(self, rid):
        """None while pending, else (x (n x nrhs), iterations, status, latency_ms)."""
        pid, nrhs = self._meta[rid]
        n = self.patterns[pid][0]
        x = np.zeros(n * nrhs)
        its = np.zeros(nrhs, np.int32)
        st = np.zeros(nrhs, np.int32)
        lat = ctypes.c_double()
        s = capi.call("culipx_server_result", self._h, int(rid), _p(x), _p(its), _p(st), ctypes.byref(lat),
                      allow=(capi.OK, capi.PENDING))
        if s == capi.PENDING:
            return None
        return x.reshape(nrhs, n).T, its, st, lat.value

    def release(self, rid):
        capi.call("culipx_server_release", self._h, int(rid))
        self._meta.pop(rid, None)

    def stats(self) -> dict:
        v = np.zeros(8, np.int64)
        capi.call("culipx_server_stats", self._h, _p(v))
        keys = ["queued", "running", "done", "batches", "running_bytes", "held_bytes", "patterns", "large_batches"]
        return {k: int(x) for k, x in zip(keys, v)}

    def launch_count(self) -> int:
        v = ctypes.c_longlong()
        capi.call("culipx_server_launch_count", self._h, ctypes.byref(v))
        return v.value

    def set_refine(self, max_refine: int, inner_tol: float = 1e-6):
        """FP64 refinement of every request to the server's tol (0: off)."""
        capi.call("culipx_server_set_refine", self._h, int(max_refine), float(inner_tol))

    def set_large_rows(self, rows: int):
        """Patterns with n >= rows are solved by the whole-GPU solver."""
        capi.call("culipx_server_set_large_rows", self._h, int(rows))

    def __del__(self):
        try:
            _release(self, "culipx_server_destroy")
        except Exception:  # interpreter shutdown
            pass


class ImportLDU:
    """ImportLDUPreconditioner: L (lower CSR), D (tri, is_piv), perm, scale as
    torch CUDA tensors (copied at creation)."""

    def __init__(self, handle: Handle, L_rowptr, L_colidx, L_val, tri, is_piv, perm, scale):
        self.handle = handle
        self.n = L_rowptr.numel() - 1
        P = ctypes.c_void_p()
        capi.call("culipx_ldu_create", handle._h, self.n, _dptr(L_rowptr), _dptr(L_colidx), _dptr(L_val), _dptr(tri),
                  _dptr(is_piv), _dptr(perm), _dptr(scale), ctypes.byref(P))
        self._h = P

    def apply(self, stage, b, x):
        capi.call("culipx_ldu_apply", self._h, int(stage), _dptr(b), _dptr(x))
        return x

    def sqmr_solve(self, A: "CsrOperator", b, x, tol=1e-8, max_it=1000):
        """Returns (residual, iterations, status)."""
        res = ctypes.c_double()
        its = ctypes.c_int()
        st = capi.call("culipx_sqmr_solve_ldu", self.handle._h, A._h, self._h, _dptr(b), _dptr(x), float(tol),
                       int(max_it), ctypes.byref(res), ctypes.byref(its), allow=(capi.OK, capi.MAXIT))
        return res.value, its.value, st

    def __del__(self):
        try:
            _release(self, "culipx_ldu_destroy")
        except Exception:  # interpreter shutdown
            pass


class KktOperator:
    """AugmentedMatrixSPMV / NormalMatrixSPMV (FP64): A is the m x n
    constraint matrix (torch CUDA CSR arrays), d the diagonal D (n), ix the
    constraint rows that get delta (torch int32 CUDA tensor or None)."""

    AUGMENTED, NORMAL = 0, 1

    def __init__(self, handle: Handle, kind, m, n, rowptr, colidx, val, d, delta=0.0, ix=None):
        self.handle = handle
        self._keep = (rowptr, colidx, val, d, ix)
        self.kind, self.m, self.n = kind, m, n
        op = ctypes.c_void_p()
        capi.call("culipx_kkt_operator_create", handle._h, int(kind), int(m), int(n), int(colidx.numel()),
                  _dptr(rowptr), _dptr(colidx), _dptr(val), _dptr(d), float(delta),
                  0 if ix is None else int(ix.numel()), None if ix is None else _dptr(ix), ctypes.byref(op))
        self._h = op

    def multiply(self, x, y, alpha=1.0, beta=0.0):
        capi.call("culipx_kkt_operator_multiply", self._h, _dptr(x), _dptr(y), float(alpha), float(beta))
        return y

    def __del__(self):
        try:
            _release(self, "culipx_kkt_operator_destroy")
        except Exception:  # interpreter shutdown
            pass


def tune_kkt_block(handle: Handle, n, m, rowptr, colidx, vals, b, precision=F32, candidates=(8, 16, 24, 32),
                   tol=1e-8, max_it=1000):
    """Block size for culipx_kkt_blocking of this KKT pattern (n H rows, m
    constraint rows): vals, b torch float64 CUDA tensors, rowptr / colidx host
    arrays.  Returns (best_block, {block: (ms, iterations, status, residual)})."""
    rp = np.ascontiguousarray(rowptr, np.int32)
    ci = np.ascontiguousarray(colidx, np.int32)
    cand = np.ascontiguousarray(candidates, np.int32)
    k = len(cand)
    ms, its, st, res = np.zeros(k), np.zeros(k, np.int32), np.zeros(k, np.int32), np.zeros(k)
    best = ctypes.c_int()
    capi.call("culipx_tune_kkt_block", handle._h, int(n), int(m), _p(rp), _p(ci), _dptr(vals), _dptr(b),
              int(precision), _p(cand), k, float(tol), int(max_it), ctypes.byref(best), _p(ms), _p(its), _p(st),
              _p(res))
    return best.value, {int(c): (float(ms[i]), int(its[i]), int(st[i]), float(res[i])) for i, c in enumerate(cand)}


def sqmr_solve_multi(handle: Handle, A: CsrOperator, M: Factor, B, X, tol=1e-8, max_it=1000):
    """Several right-hand sides of one system: B, X torch float64 CUDA tensors
    of shape (nrhs, n) (row k = right-hand side k, i.e. n x nrhs column-major).
    Returns per-RHS (residual, iterations, status) numpy arrays."""
    nrhs = int(B.shape[0])
    res = np.zeros(nrhs)
    its = np.zeros(nrhs, np.int32)
    st = np.zeros(nrhs, np.int32)
    capi.call("culipx_sqmr_solve_multi", handle._h, A._h, M._h, nrhs, _dptr(B), _dptr(X), float(tol), int(max_it),
              _p(res), _p(its), _p(st))
    return res, its, st


def sqmr_refine_multi(handle: Handle, A: CsrOperator, M: Factor, B, X, tol=1e-8, inner_tol=1e-6, inner_max_it=1000,
                      max_refine=20):
    """sqmr_refine for several right-hand sides: B, X torch float64 CUDA
    tensors of shape (nrhs, n).  Returns per-RHS (relres, iterations,
    corrections, status) numpy arrays."""
    nrhs = int(B.shape[0])
    rel = np.zeros(nrhs)
    its = np.zeros(nrhs, np.int32)
    steps = np.zeros(nrhs, np.int32)
    st = np.zeros(nrhs, np.int32)
    capi.call("culipx_sqmr_refine_multi", handle._h, A._h, M._h, nrhs, _dptr(B), _dptr(X), float(tol),
              float(inner_tol), int(inner_max_it), int(max_refine), _p(rel), _p(its), _p(steps), _p(st))
    return rel, its, steps, st


def sqmr_solve_many(handle: Handle, As, Ms, bs, xs, tol=1e-8, max_it=1000):
    """Independent systems with their own factors, one launch; per-system
    (residual, iterations, status) numpy arrays."""
    num = len(As)
    arr = lambda objs: (ctypes.c_void_p * num)(*[o._h.value if hasattr(o, "_h") else o for o in objs])
    res = np.zeros(num)
    its = np.zeros(num, np.int32)
    st = np.zeros(num, np.int32)
    capi.call("culipx_sqmr_solve_many", handle._h, num, arr(As), arr(Ms), arr([t.data_ptr() for t in bs]),
              arr([t.data_ptr() for t in xs]), float(tol), int(max_it), _p(res), _p(its), _p(st))
    return res, its, st


def batch_sqmr_refine(batch: Batch, A: CsrOperator, M: Factor, b, x, tol=1e-8, inner_tol=1e-6, inner_max_it=1000,
                      max_refine=20):
    """Per-system (relres, iterations, corrections, status) numpy arrays."""
    rel = np.zeros(batch.num)
    its = np.zeros(batch.num, np.int32)
    steps = np.zeros(batch.num, np.int32)
    st = np.zeros(batch.num, np.int32)
    capi.call("culipx_batch_sqmr_refine", batch._h, A._h, M._h, _dptr(b), _dptr(x), float(tol), float(inner_tol),
              int(inner_max_it), int(max_refine), _p(rel), _p(its), _p(steps), _p(st))
    return rel, its, steps, st


def sqmr_refine(handle: Handle, A: CsrOperator, M: Factor, b, x, tol=1e-8, inner_tol=1e-6, inner_max_it=1000,
                max_refine=20):
    """FP64 iterative refinement around SQMR (mixed precision with an FP32
    factor).  Returns (relres, total SQMR iterations, corrections, status);
    status is OK, MAXIT or STALLED (two corrections in a row did not lower
    the true residual); x is the iterate of smallest residual."""
    rel = ctypes.c_double()
    its = ctypes.c_int()
    steps = ctypes.c_int()
    st = capi.call("culipx_sqmr_refine", handle._h, A._h, M._h, _dptr(b), _dptr(x), float(tol), float(inner_tol),
                   int(inner_max_it), int(max_refine), ctypes.byref(rel), ctypes.byref(its), ctypes.byref(steps),
                   allow=(capi.OK, capi.MAXIT, capi.STALLED))
    return rel.value, its.value, steps.value, st


def sqmr_solve_noalloc(handle: Handle, A: CsrOperator, M: Factor, b, x, tol=1e-8, max_it=1000):
    """sqmr_solve without device allocation, for callers that cannot allocate
    device memory while they solve (GPU memory owned by another allocator, or
    request loops where cudaMalloc could synchronize the device).  Uses a fixed
    scratch compiled into the library: n <= 65536, one call at a time on the
    GPU.  Returns (residual, iterations, status)."""
    res = ctypes.c_double()
    its = ctypes.c_int()
    st = capi.call("culipx_sqmr_solve_noalloc", handle._h, A._h, M._h, _dptr(b), _dptr(x), float(tol), int(max_it),
                   ctypes.byref(res), ctypes.byref(its), allow=(capi.OK, capi.MAXIT))
    return res.value, its.value, st


# --------------------------------------------------------------------------
# Reference-named facade (same names, argument meaning and return values)



class BlockiLDLt:
    """BlockiLDLt<T, BK, Rook>(handle, h_A, num_pivs, piv_starts, num_blocks, block_starts).

    h_A is a host CSR triple (rowptr, colidx, val); piv_starts lists the rows
    where a pivot starts (num_pivs entries, as apps/block_ildlt builds it from
    the is_piv file); pivot is PIV_STATIC / PIV_BK / PIV_ROOK (the template
    flags); precision F64 / F32 (T).
    """

    def __init__(self, handle: Handle, h_A, num_pivs, piv_starts, num_blocks, block_starts, pivot=PIV_BK,
                 precision=F64):
        self.handle = handle
        self.rowptr, self.colidx, self.val = (np.ascontiguousarray(h_A[0], np.int32),
                                              np.ascontiguousarray(h_A[1], np.int32),
                                              np.ascontiguousarray(h_A[2], np.float64))
        self.n_ = len(self.rowptr) - 1
        self.block_starts = np.ascontiguousarray(block_starts[:num_blocks], np.int32)
        self.is_piv = np.zeros(self.n_, np.int32)
        self.is_piv[np.asarray(piv_starts[:num_pivs], dtype=np.int64)] = 1
        self.pivot = pivot
        self.precision = precision
        self.pattern = None
        self.factor = None
        self.algorithm = SOLVE_BLOCK
        self.jacobi_sweeps = 0

    def n(self):
        return self.n_

    def compute(self, fill_level, fill_factor, threshold):
        self.pattern = Pattern(self.handle, self.rowptr, self.colidx, self.block_starts, fill_level,
                               max(1.0, float(fill_factor)), self.precision)
        self.factor = Factor(self.pattern)
        self.factor.set_solve_algorithm(self.algorithm, self.jacobi_sweeps)
        self.factor.compute(self.val, self.is_piv, self.pivot, threshold)
        return 0

    def is_left(self):
        return True

    def is_middle(self):
        return True

    def is_right(self):
        return True

    def set_solve_algorithm(self, algorithm, num_jacobi_sweeps=0):
        """SOLVE_STRIPE / SOLVE_BLOCK / SOLVE_SCALAR: exact block triangular
        solves (one level-scheduled implementation); SOLVE_JACOBI: that many
        block-Jacobi sweeps per triangular solve."""
        self.algorithm = int(algorithm)
        self.jacobi_sweeps = int(num_jacobi_sweeps)
        if self.factor is not None:
            self.factor.set_solve_algorithm(self.algorithm, self.jacobi_sweeps)

    def solve_analysis(self):
        # the sweep structures are built with the factor
        return None

    def solve_left(self, b, x, transpose=False):
        return self.factor.apply(RIGHT if transpose else LEFT, b, x)

    def solve_middle(self, b, x, transpose=False):
        return self.factor.apply(MIDDLE, b, x)

    def solve_right(self, b, x, transpose=False):
        return self.factor.apply(LEFT if transpose else RIGHT, b, x)

    def export_factorized(self) -> dict:
        return self.factor.export()


class CSRMatrixSPMV:
    """CSRMatrixSPMV<T>(handle, A, explicit_At): b = alpha op(A) x + beta b."""

    def __init__(self, handle: Handle, A: CsrOperator | tuple, explicit_At=False):
        if isinstance(A, tuple):
            A = CsrOperator(handle, *A, explicit_transpose=explicit_At)
        self.A = A

    def m(self):
        return self.A.m

    def n(self):
        return self.A.n

    def multiply(self, x, b, alpha=1.0, beta=0.0, transpose=False):
        return self.A.spmv(x, b, alpha, beta, transpose)


class SQMR:
    """SQMR<T>(handle, spmv, tol, max_it, prec).solve(b, x) -> (residual, iterations)."""

    def __init__(self, handle: Handle, spmv: CSRMatrixSPMV, tol, max_it, preconditioner: BlockiLDLt | None = None):
        self.handle, self.spmv, self.tol, self.max_it, self.prec = handle, spmv, tol, max_it, preconditioner

    def solve(self, b, x):
        M = self.prec.factor if self.prec is not None else None
        res, its, _ = sqmr_solve(self.handle, self.spmv.A, M, b, x, self.tol, self.max_it)
        return res, its
