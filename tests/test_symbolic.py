"""Symbolic analysis: the product's C++ analysis (host-only handle) must equal
the oracle's restatement of the reference's host phase bit for bit:
coarse pattern, level fill, levels (rows ascending per level), factor-order
and U'-sweep block lists, block formats and max_nnz."""
import ctypes

import numpy as np
import pytest

import culip_b200 as cb
from culip_b200 import _capi as capi
import oracle
from problems import kkt, permute_sym, random_blocking, random_spd_ish, scrambled_kkt


class HostHandle:
    def __init__(self):
        h = ctypes.c_void_p()
        capi.call("culipx_handle_create", ctypes.byref(h), -1, None)
        self._h = h

    def __del__(self):
        capi.load().culipx_handle_destroy(self._h)


@pytest.fixture(scope="module")
def hh():
    return HostHandle()


def _compare(hh, rp, ci, bs, fill_level, fill_factor=1.0, precision=cb.F64):
    dt = np.float64 if precision == cb.F64 else np.float32
    S = oracle.Sym(rp, ci, bs, fill_level, fill_factor, dtype=dt)
    P = cb.Pattern(hh, rp, ci, bs, fill_level, fill_factor, precision)
    E = P.export()
    inf = P.info()
    assert inf["coarse_nnz"] == S.coarse_nnz and inf["num_levels"] == S.num_levels
    assert inf["fill_nnz"] == S.fill_nnz
    pairs = [("coarse_off", S.cs_off), ("coarse_col", S.cs_col), ("blk_nnzA", S.blk_nnzA), ("lvl_off", S.lvl_off),
             ("lvl_rows", S.lvl_rows), ("lb_off", S.lb_off), ("lb", S.lb), ("sb_off", S.sb_off), ("sb", S.sb),
             ("fmt", S.fmt), ("max_nnz", S.max_nnz)]
    for k, ref in pairs:
        assert np.array_equal(E[k], ref), k
    return S, E


@pytest.mark.parametrize("precision", [cb.F64, cb.F32])
def test_small_kkt(hh, precision):
    rp, ci, v, bs = kkt("small")
    S, E = _compare(hh, rp, ci, bs, 0, precision=precision)
    # natural-order KKT with level-0 fill: two levels (H rows, then A rows)
    assert S.num_levels == 2


@pytest.mark.parametrize("seed", [7, 8, 9])
@pytest.mark.parametrize("fill_level", [0, 1, 2, 3])
def test_scrambled(hh, seed, fill_level):
    rp, ci, v, bs = scrambled_kkt(seed=seed)
    _compare(hh, rp, ci, bs, fill_level)


@pytest.mark.parametrize("fill_factor", [1.0, 1.7, 4.0])
def test_fill_factor_and_formats(hh, fill_factor):
    rp, ci, v, bs = scrambled_kkt(seed=11, block_lo=8, block_hi=32)
    S, E = _compare(hh, rp, ci, bs, 1, fill_factor)
    assert (S.fmt == 0).any() and (S.fmt == 1).any()


def test_random_symmetric_odd_blocks(hh):
    rp, ci, v = random_spd_ish(700, 0.01)
    bs = random_blocking(700, np.random.default_rng(1), 1, 32)
    _compare(hh, rp, ci, bs, 2)


def test_missing_diagonal_blocks_are_added(hh):
    # a matrix whose diagonal blocks have no entries of their own
    n = 64
    rows, cols = [], []
    for i in range(n):
        j = (i + 17) % n
        rows += [i, j]
        cols += [j, i]
    import scipy.sparse as sp

    A = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n))
    A.sum_duplicates()
    A.sort_indices()
    bs = np.arange(0, n + 1, 8, dtype=np.int32)
    S, E = _compare(hh, A.indptr.astype(np.int32), A.indices.astype(np.int32), bs, 0)
    assert S.fill_nnz > 0


def test_rejects_bad_input(hh):
    rp, ci, v, bs = kkt("small")
    with pytest.raises(cb.CulipxError):
        cb.Pattern(hh, rp, ci, bs, 0, 0.5)  # fill_factor < 1
    bad = bs.copy()
    bad[1] = 40  # block of 40 rows
    with pytest.raises(cb.CulipxError):
        cb.Pattern(hh, rp, ci, bad, 0, 1.0)
    ci2 = ci.copy()
    ci2[0], ci2[1] = ci2[1], ci2[0]  # unsorted row
    with pytest.raises(cb.CulipxError):
        cb.Pattern(hh, rp, ci2, bs, 0, 1.0)


def test_generator_properties():
    cfg = cb.KKT_CONFIGS["small"]
    rp, ci, v = cb.kkt_generate(3000, 1500, 6, 32, 1e-6, 1e6)
    import scipy.sparse as sp

    N = 4500
    K = sp.csr_matrix((v, ci, rp), shape=(N, N))
    assert abs(K - K.T).max() == 0
    assert len(ci) == N + 2 * 3000 * 6
    assert np.all(np.diff(ci[rp[0]:rp[1]]) > 0)
    d = K.diagonal()
    assert np.all(d[:3000] > 0) and np.allclose(d[3000:], -1e-8)
    # half of each column inside the band around floor(j m / n)
    A = K[3000:, :3000].tocsc()
    j = np.arange(3000)
    center = j * 1500 // 3000
    rows = [A.indices[A.indptr[c]:A.indptr[c + 1]] for c in range(3000)]
    inband = np.array([np.sum(np.abs(r - center[c] + 0.5) <= 32) for c, r in enumerate(rows)])
    assert np.all(inband >= 3)
    # determinism
    rp2, ci2, v2 = cb.kkt_generate(3000, 1500, 6, 32, 1e-6, 1e6)
    assert np.array_equal(v, v2) and np.array_equal(ci, ci2)


def test_blocking_rule():
    bs = cb.kkt_blocking(200000, 100000, 32)
    assert bs[-1] == 300000 and 200000 in bs
    sizes = np.diff(bs)
    assert sizes.min() >= 8 and sizes.max() <= 32
    bs = cb.kkt_blocking(1003, 517, 32)
    sizes = np.diff(bs)
    assert 1003 in bs and sizes.min() >= 8 and sizes.max() <= 32


def test_permute_helper_roundtrip():
    rp, ci, v, bs = kkt("small")
    perm = np.random.default_rng(0).permutation(len(rp) - 1)
    rp2, ci2, v2 = permute_sym(rp, ci, v, perm)
    import scipy.sparse as sp

    K = sp.csr_matrix((v, ci, rp))
    K2 = sp.csr_matrix((v2, ci2, rp2))
    assert abs(K[perm][:, perm] - K2).max() == 0
