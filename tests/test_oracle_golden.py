"""Pins the CPU oracle to the reference's own golden fixtures and assertions.

tests/la/test_sqmr.cc:192-293: SQMR on sqmr_{small,big}_A with x = 1, b = A x,
with and without the imported L D L' preconditioner (L, D in 1x1/2x2 blocks,
permutation p, scaling s); asserts ||b - A x|| <= test_tol ||b|| and
iterations <= n (double: term_tol 1e-10, test_tol 1e-5).
tests/la/test_spmv.cc:150-168: CSR SpMV on spmv_A / spmv_K with x = 0.1,
A x and A' x against cuSPARSE within 1e-10 (double); scipy stands in for
cuSPARSE here.
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


def tridiag_from_D(rowptr, colidx, val, n):
    """The conversion of tests/la/test_sqmr.cc:103-152 (csr D -> [sup, diag, sub] + is_piv)."""
    tri = np.zeros(3 * n)
    is_piv = np.ones(n, np.int32)
    i = 0
    while i < n:
        ln = rowptr[i + 1] - rowptr[i]
        iv = val[rowptr[i]:rowptr[i + 1]]
        if ln == 1:
            if i > 0:
                tri[3 * (i - 1) + 2] = 0
            tri[3 * i + 1] = iv[0]
            if i < n - 1:
                tri[3 * (i + 1)] = 0
            i += 1
        else:
            ipv = val[rowptr[i + 1]:rowptr[i + 2]]
            tri[3 * i] = 0
            tri[3 * i + 1] = iv[0]
            tri[3 * i + 2] = iv[1]
            tri[3 * (i + 1)] = ipv[0]
            tri[3 * (i + 1) + 1] = ipv[1]
            tri[3 * (i + 1) + 2] = 0
            is_piv[i + 1] = 0
            i += 2
    return tri, is_piv


@pytest.mark.parametrize("case,precondition", [("small", False), ("small", True), ("big", True)])
def test_sqmr_reference_fixture(case, precondition):
    d = _load(f"sqmr_{case}.npz")
    rp, ci, v = d["A_rowptr"], d["A_colidx"], d["A_val"]
    n = len(rp) - 1
    A = sp.csr_matrix((v, ci, rp), shape=(n, n))
    xt = np.ones(n)
    b = A @ xt
    term_tol, test_tol = 1e-10, 1e-5
    if precondition:
        # the fixture's D is stored symmetric: expand like Test<T>::read_matrix_csr
        tri, is_piv = tridiag_from_D(d["D_rowptr"], d["D_colidx"], d["D_val"], n)
        x, res, it = oracle.sqmr_ldu(rp, ci, v, d["L_rowptr"], d["L_colidx"], d["L_val"], tri, is_piv, d["perm"],
                                     d["scale"], b, term_tol, n)
    else:
        x, res, it = oracle.sqmr(rp, ci, v, b, None, term_tol, n)
    real_res = np.linalg.norm(b - A @ x)
    assert real_res <= test_tol * np.linalg.norm(b)
    assert it <= n


@pytest.mark.parametrize("name", ["A", "K"])
@pytest.mark.parametrize("transpose", [False, True])
def test_spmv_reference_fixture(name, transpose):
    d = _load(f"spmv_{name}.npz")
    m, n = int(d["m"]), int(d["n"])
    A = sp.csr_matrix((d["val"], d["colidx"], d["rowptr"]), shape=(m, n))
    if transpose:
        At = A.T.tocsr()
        At.sort_indices()
        rp, ci, v = At.indptr, At.indices, At.data
        x = np.full(m, 0.1)
        ref = A.T @ x
    else:
        rp, ci, v = d["rowptr"], d["colidx"], d["val"]
        x = np.full(n, 0.1)
        ref = A @ x
    y = oracle.spmv(rp, ci, v, x)
    assert np.allclose(y, ref, rtol=1e-10, atol=1e-10)
