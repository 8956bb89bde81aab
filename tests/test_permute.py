"""Permutation / scaling of K before the factorization (T_matrix_permute_scale,
libs/la/sparse_la.impl.cuh:599-657, as called by the driver's host_permute,
apps/block_ildlt/block_ildlt_invariants.h:31-69).

CPU: the oracle's restatement against P A P' computed densely, the
new -> old convention, both scaling modes, and the C ABI's argument checks.
GPU: the plan + gather kernels against the oracle, bit for bit (structure and
values), FP64 and FP32, symmetric and two-sided permutations."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import culip_b200 as cb
from culip_b200 import _capi as capi
import oracle
from problems import kkt


def _random_csr(n, density, seed, dtype=np.float64, symmetric=True):
    rng = np.random.default_rng(seed)
    A = sp.random(n, n, density=density, random_state=rng, format="csr")
    if symmetric:
        A = A + A.T
    A = A + sp.eye(n)
    A = A.tocsr()
    A.sort_indices()
    return A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(dtype)


def _dense(rp, ci, v, n):
    return sp.csr_matrix((v, ci, rp), shape=(n, n)).toarray()


@pytest.mark.parametrize("old_to_new", [True, False])
def test_oracle_matches_dense_permutation(old_to_new):
    n = 60
    rp, ci, v = _random_csr(n, 0.08, 3)
    p = np.random.default_rng(4).permutation(n)
    B = oracle.permute_scale(rp, ci, v, p, perm_is_old_to_new=old_to_new)
    fwd = p if old_to_new else np.argsort(p)
    P = np.zeros((n, n))
    P[fwd, np.arange(n)] = 1.0
    assert np.array_equal(_dense(*B, n), P @ _dense(rp, ci, v, n) @ P.T)
    # rows and columns sorted
    for i in range(n):
        assert np.all(np.diff(B[1][B[0][i]:B[0][i + 1]]) > 0)


@pytest.mark.parametrize("before", [True, False])
def test_oracle_scaling(before):
    n = 40
    rp, ci, v = _random_csr(n, 0.1, 5)
    rng = np.random.default_rng(6)
    p = rng.permutation(n)
    r = rng.uniform(0.5, 2.0, n)
    c = rng.uniform(0.5, 2.0, n)
    B = oracle.permute_scale(rp, ci, v, p, row_scale=r, col_scale=c, scale_before_match=before)
    rows = np.repeat(np.arange(n), np.diff(rp))
    s = r[rows] * c[ci] if before else r[p[rows]] * c[p[ci]]
    expect = oracle.permute_scale(rp, ci, v / s, p)
    assert np.array_equal(B[2], expect[2])


def test_capi_rejects_bad_permutation():
    h = ctypes.c_void_p()
    capi.call("culipx_handle_create", ctypes.byref(h), -1, None)
    try:
        perm = np.array([0, 0, 1], np.int32)
        out = ctypes.c_void_p()
        st = capi.load().culipx_permute_create(h, 3, 5, ctypes.c_void_p(16), ctypes.c_void_p(16),
                                               perm.ctypes.data_as(ctypes.c_void_p), None, 1, ctypes.byref(out))
        assert st == capi.INVALID_ARG
        assert b"permutation" in capi.load().culipx_last_error()
        perm = np.array([0, 3, 1], np.int32)
        st = capi.load().culipx_permute_create(h, 3, 5, ctypes.c_void_p(16), ctypes.c_void_p(16),
                                               perm.ctypes.data_as(ctypes.c_void_p), None, 1, ctypes.byref(out))
        assert st == capi.INVALID_ARG
    finally:
        capi.load().culipx_handle_destroy(h)


def _gpu_case(rp, ci, v, row_perm, col_perm=None, old_to_new=True, scales=None, before=False):
    import torch

    h = cb.Handle(0)
    d_rp = torch.from_numpy(rp).cuda()
    d_ci = torch.from_numpy(ci).cuda()
    d_v = torch.from_numpy(v).cuda()
    plan = cb.PermutePlan(h, d_rp, d_ci, row_perm, col_perm, old_to_new)
    out = torch.empty_like(d_v)
    rs = cs = None
    if scales is not None:
        rs = torch.from_numpy(scales[0].astype(v.dtype)).cuda()
        cs = torch.from_numpy(scales[1].astype(v.dtype)).cuda()
    plan.apply(d_v, out, rs, cs, before)
    torch.cuda.synchronize()
    b_rp, b_ci = plan.structure()
    ref = oracle.permute_scale(rp, ci, v, row_perm, col_perm,
                               None if scales is None else scales[0].astype(v.dtype),
                               None if scales is None else scales[1].astype(v.dtype), before, old_to_new)
    assert np.array_equal(b_rp, ref[0])
    assert np.array_equal(b_ci, ref[1])
    assert np.array_equal(out.cpu().numpy(), ref[2])


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("old_to_new", [True, False])
def test_gpu_symmetric_permutation(dtype, old_to_new):
    rp, ci, v = _random_csr(2000, 0.004, 11, dtype)
    p = np.random.default_rng(12).permutation(2000).astype(np.int32)
    _gpu_case(rp, ci, v, p, None, old_to_new)


@pytest.mark.gpu
@pytest.mark.parametrize("before", [True, False])
def test_gpu_two_sided_scaled(before):
    rp, ci, v = _random_csr(1500, 0.005, 13, symmetric=False)
    rng = np.random.default_rng(14)
    pr = rng.permutation(1500).astype(np.int32)
    pc = rng.permutation(1500).astype(np.int32)
    scales = (rng.uniform(0.25, 4.0, 1500), rng.uniform(0.25, 4.0, 1500))
    _gpu_case(rp, ci, v, pr, pc, True, scales, before)


@pytest.mark.gpu
def test_gpu_kkt_long_rows_and_identity():
    rp, ci, v, _ = kkt("small")
    n = len(rp) - 1
    _gpu_case(rp, ci, v, np.arange(n, dtype=np.int32))
    # a row longer than a warp: dense first row / column
    m = 100
    A = sp.lil_matrix((m, m))
    A[0, :] = np.arange(1, m + 1)
    A[:, 0] = np.arange(1, m + 1)[:, None]
    A.setdiag(7.0)
    A = A.tocsr()
    A.sort_indices()
    p = np.random.default_rng(15).permutation(m).astype(np.int32)
    _gpu_case(A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64), p)
