"""Algebraic checks of the oracle's restatement (independent of any GPU):

* zero-skipping Schur products equal the literal dense 32x32x32 tile
  products of the reference (d_apply_left_right_update) bit for bit;
* with complete fill (level of fill >= the depth of the elimination, no
  threshold, fill_factor large enough to keep every block entry) the
  incomplete factor is exact: U'^-1 P' K P U^-1 = D.
"""
import numpy as np
import pytest

import culip_b200 as cb
import oracle
from problems import kkt, scrambled_kkt


@pytest.mark.parametrize("seed,fill", [(7, 0), (8, 1), (9, 2)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_literal_equals_sparse_products(seed, fill, dtype):
    rp, ci, v, bs = scrambled_kkt(seed=seed)
    S = oracle.Sym(rp, ci, bs, fill, 1.0, dtype=dtype)
    a = S.factor(v.astype(dtype)).export()
    b = S.factor(v.astype(dtype), literal=True).export()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("pivot", [cb.PIV_BK, cb.PIV_ROOK, cb.PIV_STATIC])
@pytest.mark.parametrize("case", ["indefinite", "kkt"])
def test_complete_factorization_is_exact(pivot, case):
    """Pivoting stays inside diagonal blocks, so exactness is checked on
    orderings whose block pivots are well conditioned (a scrambled KKT can put
    a -gamma = -1e-8 row first and then loses ~1e8 in accuracy by design)."""
    if case == "indefinite":
        from problems import random_blocking, random_spd_ish

        rp, ci, v = random_spd_ish(240, 0.03, seed=4)
        bs = random_blocking(240, np.random.default_rng(2), 3, 12)
    else:
        rp, ci, v = cb.kkt_generate(120, 60, 3, 0, 1e-1, 1e1)
        bs = cb.kkt_blocking(120, 60, 6)
    n = len(rp) - 1
    S = oracle.Sym(rp, ci, bs, 10 ** 6, 1024.0)
    F = S.factor(v, pivot=pivot)
    import scipy.sparse as sp

    K = sp.csr_matrix((v, ci, rp), shape=(n, n))
    rng = np.random.default_rng(0)
    for _ in range(3):
        y = rng.standard_normal(n)
        z = F.apply(cb.LEFT, K @ F.apply(cb.RIGHT, y))
        dy = F.apply(cb.MIDDLE, z)  # D^-1 (U'^-1 P' K P U^-1) y == y
        assert np.linalg.norm(dy - y) <= 1e-10 * np.linalg.norm(y)


def test_natural_kkt_two_levels_and_identity_h_blocks():
    rp, ci, v, bs = kkt("small")
    S = oracle.Sym(rp, ci, bs, 0, 1.0)
    E = S.factor(v).export()
    # H rows (level 0): pivot tiles are exactly the identity, D = H + delta
    nH = 2000
    tri = E["tri"].reshape(-1, 3)
    assert np.array_equal(tri[:nH, 1], v[np.asarray([np.searchsorted(ci[rp[i]:rp[i + 1]], i) + rp[i]
                                                     for i in range(nH)])])
    assert np.all(tri[:nH, 0] == 0) and np.all(tri[:nH, 2] == 0)


def test_kkt_operator_restatement_algebra():
    """The augmented operator is K = [[D, A'], [A, shift]] times x, and the
    normal operator equals its Schur complement form A D^-1 A' x + shift x."""
    import scipy.sparse as sp

    rng = np.random.default_rng(9)
    n, m = 60, 25
    A = sp.random(m, n, density=0.1, random_state=3, format="csr")
    d = 10.0 ** rng.uniform(-2, 2, n)
    ix = np.array([0, 4, 7, 24])
    x = rng.standard_normal(n + m)
    shift = np.zeros(m)
    shift[ix] = 0.3
    K = sp.bmat([[sp.diags(d), A.T], [A, sp.diags(shift)]]).tocsr()
    got = oracle.kkt_operator(0, A.indptr, A.indices, A.data, n, d, x, 0.3, ix)
    assert np.allclose(got, K @ x, rtol=1e-14, atol=1e-14)
    xm = x[:m]
    want = A @ (A.T @ xm / d) + shift * xm
    assert np.allclose(oracle.kkt_operator(1, A.indptr, A.indices, A.data, n, d, xm, 0.3, ix), want, rtol=1e-14)
