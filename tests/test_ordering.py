"""Orderings: culipx_sprank (culip's sprank, libs/algorithms/sprank.cuh) and
culipx_ordering_rcm.

The structural rank is pinned by the reference's own fixtures and bounds
(tests/algorithms/test_bound_rank.cc:84-86: sprank = the upper bound 800, 930,
4380), converted by tests/golden/make_fixtures.py, and checked against scipy's
maximum bipartite matching on random patterns.  The RCM ordering is checked as
a permutation, for determinism, and by the bandwidth it recovers from a
scrambled banded pattern; on the GPU, an RCM-ordered KKT system runs through the
permutation plan, the factor and the applies (bit-exact against the oracle)
and SQMR."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import maximum_bipartite_matching

import culip_b200 as cb

HERE = os.path.dirname(os.path.abspath(__file__))
INT_MAX = 2**31 - 1


def _check_matching(m, n, rp, ci, rank, rmatch, cmatch):
    rows = np.repeat(np.arange(m), np.diff(rp))
    entries = set(zip(rows.tolist(), ci.tolist()))
    matched = [(i, int(j)) for i, j in enumerate(rmatch) if j != INT_MAX]
    assert len(matched) == rank
    assert all(e in entries for e in matched)
    assert all(cmatch[j] == i for i, j in matched)
    assert np.sum(cmatch != INT_MAX) == rank


@pytest.mark.parametrize("name", ["bound_rank_51_800", "bound_rank_920_930", "bound_rank_4380_4380"])
def test_sprank_reference_fixtures(name):
    f = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    m, n = int(f["m"]), int(f["n"])
    rank, rmatch, cmatch = cb.sprank(m, n, f["rowptr"], f["colidx"])
    assert rank == int(f["ub"])
    _check_matching(m, n, f["rowptr"], f["colidx"], rank, rmatch, cmatch)


@pytest.mark.parametrize("seed", range(6))
def test_sprank_matches_scipy_maximum_matching(seed):
    rng = np.random.default_rng(seed)
    m, n = int(rng.integers(1, 300)), int(rng.integers(1, 300))
    A = sp.random(m, n, density=float(rng.uniform(0.002, 0.03)), format="csr", random_state=seed)
    A.sort_indices()
    rp, ci = A.indptr.astype(np.int32), A.indices.astype(np.int32)
    rank, rmatch, cmatch = cb.sprank(m, n, rp, ci)
    want = int(np.sum(maximum_bipartite_matching(A, perm_type="column") >= 0))
    assert rank == want
    _check_matching(m, n, rp, ci, rank, rmatch, cmatch)


def test_sprank_edge_cases():
    assert cb.sprank(0, 0, np.zeros(1, np.int32), np.zeros(0, np.int32))[0] == 0
    rp = np.array([0, 0, 2, 2], np.int32)  # empty first and last rows
    rank, rmatch, cmatch = cb.sprank(3, 2, rp, np.array([0, 1], np.int32))
    assert rank == 1 and rmatch[0] == INT_MAX and rmatch[2] == INT_MAX
    with pytest.raises(cb.CulipxError):
        cb.sprank(2, 2, np.array([0, 1, 2], np.int32), np.array([0, 5], np.int32))


def _bandwidth(rp, ci):
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    return int(np.max(np.abs(rows - ci))) if len(ci) else 0


def _permute(rp, ci, perm):
    """B = P A P' with perm[new] = old."""
    n = len(rp) - 1
    inv = np.empty(n, np.int64)
    inv[perm] = np.arange(n)
    A = sp.csr_matrix((np.ones(len(ci)), ci, rp), shape=(n, n))
    B = A[perm][:, perm].tocsr()
    B.sort_indices()
    return B.indptr.astype(np.int32), B.indices.astype(np.int32)


def test_rcm_recovers_a_scrambled_band():
    rng = np.random.default_rng(1)
    n, half = 2000, 5
    A = sp.diags([np.ones(n - abs(k)) for k in range(-half, half + 1)], list(range(-half, half + 1)), format="csr")
    scr = rng.permutation(n).astype(np.int32)
    rp, ci = _permute(A.indptr.astype(np.int32), A.indices.astype(np.int32), scr)
    assert _bandwidth(rp, ci) > 500
    perm = cb.ordering_rcm(rp, ci)
    assert np.array_equal(np.sort(perm), np.arange(n))
    assert np.array_equal(perm, cb.ordering_rcm(rp, ci))
    brp, bci = _permute(rp, ci, perm)
    assert _bandwidth(brp, bci) <= 2 * half


def test_rcm_components_and_isolated_vertices():
    # two components and isolated vertices, an unsymmetric pattern is symmetrized
    rp = np.array([0, 1, 2, 2, 3, 3, 3], np.int32)
    ci = np.array([1, 3, 4], np.int32)
    perm = cb.ordering_rcm(rp, ci)
    assert np.array_equal(np.sort(perm), np.arange(6))


@pytest.mark.gpu
def test_rcm_ordered_kkt_factor_and_solve():
    """The small KKT system under its RCM ordering: permutation plan on the
    device, blocking of the permuted pattern, factor and applies bit-exact
    against the oracle, the first SQMR iterations against the oracle's."""
    torch = pytest.importorskip("torch")
    import oracle

    cfg = cb.KKT_CONFIGS["small"]
    n, m = cfg["n"], cfg["m"]
    rp, ci, v = cb.kkt_generate(n, m, cfg["nnz_per_col"], cfg["band_half"], cfg["hmin"], cfg["hmax"])
    N = n + m
    perm = cb.ordering_rcm(rp, ci)
    h = cb.Handle(0)
    plan = cb.PermutePlan(h, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), perm, perm_is_old_to_new=False)
    brp, bci = plan.structure()
    bv = torch.zeros(len(ci), dtype=torch.float64, device="cuda")
    plan.apply(torch.from_numpy(v).cuda(), bv)
    orp, oci, ov = oracle.permute_scale(rp, ci, v, perm, perm_is_old_to_new=False)
    assert np.array_equal(brp, orp) and np.array_equal(bci, oci) and np.array_equal(bv.cpu().numpy(), ov)
    bs = cb.blocking_generate(brp, bci, 8, 32)
    P = cb.Pattern(h, brp, bci, bs, 0, 1.0, cb.F64)
    F = cb.Factor(P)
    F.compute(bv)
    S = oracle.Sym(brp, bci, bs, 0, 1.0)
    E, Eo = F.export(), S.factor(ov).export()
    for k in ("blk_off", "idx", "val", "tri", "is_piv", "perm"):
        assert np.array_equal(E[k], Eo[k]), k
    OF = S.factor(ov)
    b = cb.normal_vector(cb.SEED + 1, N)
    bt = torch.from_numpy(b).cuda()
    for stage in (cb.LEFT, cb.MIDDLE, cb.RIGHT):
        assert np.array_equal(F.apply(stage, bt).cpu().numpy(), OF.apply(stage, b)), stage
    # RCM mixes H and A rows in the blocks (12 levels here) and ILDL(0) + SQMR
    # breaks down on this ordering after a few hundred iterations, at an
    # iteration that depends on rounding; compare a fixed 10 iterations
    A = cb.CsrOperator(h, torch.from_numpy(brp).cuda(), torch.from_numpy(bci).cuda(), bv)
    x = torch.zeros(N, dtype=torch.float64, device="cuda")
    res, its, _ = cb.sqmr_solve(h, A, F, bt, x, 0.0, 10)
    xo, reso, itso = oracle.sqmr(orp, oci, ov, b, OF, 0.0, 10)
    assert its == itso == 10
    assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-6 * np.linalg.norm(xo)
