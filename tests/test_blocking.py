"""The blocking generator (host code, no GPU): a partition of the rows into
contiguous blocks of at most max_size rows that keeps equal-structure runs
whole and feeds the factor like the driver's blocking files."""
import numpy as np
import pytest
import scipy.sparse as sp

import culip_b200 as cb
import oracle


def _sym_pattern(n, density, seed):
    A = sp.random(n, n, density=density, random_state=seed, format="csr")
    S = (A + A.T + sp.eye(n)).tocsr()
    S.sort_indices()
    return S.indptr.astype(np.int32), S.indices.astype(np.int32)


def _check_partition(bs, n, lo, hi):
    assert bs[0] == 0 and bs[-1] == n and np.all(np.diff(bs) > 0)
    sizes = np.diff(bs)
    assert sizes.max() <= hi
    if len(sizes) > 1:
        assert sizes[-1] >= min(lo, n)


@pytest.mark.parametrize("lo,hi", [(8, 32), (4, 16), (1, 8)])
def test_partition(lo, hi):
    rp, ci = _sym_pattern(1000, 0.004, 1)
    bs = cb.blocking_generate(rp, ci, lo, hi)
    _check_partition(bs, 1000, lo, hi)
    assert np.array_equal(bs, cb.blocking_generate(rp, ci, lo, hi))  # deterministic


def test_equal_structure_runs_stay_together():
    # rows 10..14 share one column set (a dense 5x5 block coupled to row 30)
    n = 60
    rows, cols = list(range(n)), list(range(n))
    for i in range(10, 15):
        for j in list(range(10, 15)) + [30]:
            if i != j:
                rows.append(i)
                cols.append(j)
                rows.append(j)
                cols.append(i)
    S = sp.csr_matrix((np.ones(len(rows)), (rows, cols)), shape=(n, n))
    S.sum_duplicates()
    S.sort_indices()
    bs = cb.blocking_generate(S.indptr, S.indices, 8, 32)
    _check_partition(bs, n, 8, 32)
    blk = np.searchsorted(bs, np.arange(n), side="right") - 1
    assert len(set(blk[10:15])) == 1


def test_coupled_rows_fill_a_block():
    # a dense 20-row diagonal block: one block of 20 (closing needs a run not coupled to the block)
    n = 50
    D = sp.block_diag([np.ones((20, 20)), sp.eye(30)]).tocsr()
    D.sort_indices()
    bs = cb.blocking_generate(D.indptr, D.indices, 8, 32)
    assert 20 in bs and bs[0] == 0 and np.all(np.diff(bs[: list(bs).index(20) + 1]) == 20)


def test_small_and_bad_input():
    rp, ci = _sym_pattern(5, 0.3, 2)
    assert list(cb.blocking_generate(rp, ci, 8, 32)) == [0, 5]
    with pytest.raises(cb.CulipxError):
        cb.blocking_generate(rp, ci, 16, 8)
    with pytest.raises(cb.CulipxError):
        cb.blocking_generate(rp, ci[::-1].copy(), 8, 32)


def test_generated_blocking_feeds_the_factor():
    rp, ci, v = cb.kkt_generate(2000, 1000, 4, 0, 1e-2, 1e2)
    bs = cb.blocking_generate(rp, ci, 8, 32)
    _check_partition(bs, 3000, 8, 32)
    F = oracle.Sym(rp, ci, bs, 0, 1.0).factor(v)
    b = cb.normal_vector(cb.SEED + 1, 3000)
    x, res, its = oracle.sqmr(rp, ci, v, b, F, 1e-8, 1000)
    # the stopping test passes well before max_it, as with the KKT blocking (256 iterations)
    assert its < 400
