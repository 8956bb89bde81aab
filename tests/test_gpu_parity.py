"""GPU parity: the sm_100a path through the C ABI against the CPU oracle.

Factor, D, pivots and permutation are compared exactly (the kernels and the
oracle spell out the same roundings); preconditioner applies, SpMV and SQMR
with stated tolerances.
"""
import numpy as np
import pytest

import culip_b200 as cb
from culip_b200 import _capi as capi
import oracle
from problems import kkt, random_spd_ish, scrambled_kkt

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def handle():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return cb.Handle(0)


def _factor_both(handle, rp, ci, v, bs, fill_level=0, pivot=cb.PIV_BK, precision=cb.F64, is_piv=None,
                 threshold=0.0):
    dt = np.float64 if precision == cb.F64 else np.float32
    S = oracle.Sym(rp, ci, bs, fill_level, 1.0, dtype=dt)
    OF = S.factor(v.astype(dt), is_piv=is_piv, pivot=pivot, threshold=threshold)
    P = cb.Pattern(handle, rp, ci, bs, fill_level, 1.0, precision)
    F = cb.Factor(P)
    tv = torch.from_numpy(v.astype(dt)).cuda()
    F.compute(tv, is_piv=is_piv, pivot=pivot, threshold=threshold)
    return S, OF, P, F


def _assert_factor_equal(oe, ge):
    for k in ("blk_off", "blk_nnz", "idx", "is_piv", "perm", "got_extra"):
        assert np.array_equal(oe[k], ge[k]), k
    # exact equality of every stored value (signed zeros compare equal)
    assert np.array_equal(oe["val"], ge["val"])
    assert np.array_equal(oe["tri"], ge["tri"])


@pytest.mark.parametrize("pivot", [cb.PIV_BK, cb.PIV_STATIC, cb.PIV_ROOK])
def test_factor_small_kkt_exact(handle, pivot):
    rp, ci, v, bs = kkt("small")
    S, OF, P, F = _factor_both(handle, rp, ci, v, bs, pivot=pivot)
    _assert_factor_equal(OF.export(), F.export())


@pytest.mark.parametrize("precision", [cb.F64, cb.F32])
@pytest.mark.parametrize("threshold", [0.0, 1e-3])
def test_factor_banded_b32_exact(handle, precision, threshold):
    """32-row blocks with a banded half of A: update columns of more than 32
    blocks, sparse blocks of more than 8 and of more than 32 entries (every
    path of the pivot-block updates and of the entrywise off-diagonal pass);
    with a drop threshold every off-diagonal block takes the tiled pass."""
    rp, ci, v, bs = kkt("small", block=32, band_half=16)
    S, OF, P, F = _factor_both(handle, rp, ci, v, bs, precision=precision, threshold=threshold)
    _assert_factor_equal(OF.export(), F.export())
    b = cb.normal_vector(5, len(rp) - 1)
    dt = np.float64 if precision == cb.F64 else np.float32
    for stage in (cb.LEFT, cb.MIDDLE, cb.RIGHT):
        xo = OF.apply(stage, b.astype(dt))
        xg = F.apply(stage, torch.from_numpy(b.astype(dt)).cuda()).cpu().numpy()
        assert np.array_equal(xo, xg), stage


@pytest.mark.parametrize("precision", [cb.F64, cb.F32])
@pytest.mark.parametrize("threshold", [0.0, 1e-3])
def test_factor_graph_replay_exact(handle, precision, threshold):
    """The factorization replayed from its CUDA graph equals an ordinary
    compute bit for bit, also after the values behind the pointer change."""
    rp, ci, v, bs = kkt("small")
    dt = np.float32 if precision == cb.F32 else np.float64
    P = cb.Pattern(handle, rp, ci, bs, 0, 1.0, precision)
    Fg, Fr = cb.Factor(P), cb.Factor(P)
    dv = torch.from_numpy(v.astype(dt)).cuda()
    rng = np.random.default_rng(12)
    for step in range(3):
        Fg.compute_graph(dv, cb.PIV_BK, threshold)
        Fr.compute(dv.clone(), None, cb.PIV_BK, threshold)
        eg, er = Fg.export(), Fr.export()
        for k in er:
            assert np.array_equal(eg[k], er[k]), (step, k)
        bvec = torch.from_numpy(cb.normal_vector(3 + step, len(rp) - 1).astype(dt)).cuda()
        for stage in (cb.LEFT, cb.MIDDLE, cb.RIGHT):  # the solve structures were rebuilt by the replay too
            xg, xr = torch.zeros_like(bvec), torch.zeros_like(bvec)
            Fg.apply(stage, bvec, xg)
            Fr.apply(stage, bvec, xr)
            assert torch.equal(xg, xr), (step, stage)
        # new values in the same buffer: the graph reads them on its next replay
        dv.copy_(torch.from_numpy((v * 10.0 ** rng.uniform(-0.5, 0.5, len(v))).astype(dt)))
    assert Fg.stats()[1] == Fr.stats()[1]  # the replay launches the same kernels


def test_factor_small_kkt_fp32_exact(handle):
    rp, ci, v, bs = kkt("small")
    S, OF, P, F = _factor_both(handle, rp, ci, v, bs, precision=cb.F32)
    _assert_factor_equal(OF.export(), F.export())


@pytest.mark.parametrize("seed", [7, 8])
@pytest.mark.parametrize("fill_level", [0, 1, 2])
def test_factor_scrambled_exact(handle, seed, fill_level):
    """Random symmetric permutation + random blocking: deep level schedules,
    2x2 pivots, swaps propagated to the column blocks, level fill, dual dropping."""
    rp, ci, v, bs = scrambled_kkt(seed=seed)
    S, OF, P, F = _factor_both(handle, rp, ci, v, bs, fill_level=fill_level)
    oe, ge = OF.export(), F.export()
    assert (oe["is_piv"] == 0).sum() > 0  # the case exercises 2x2 pivots
    _assert_factor_equal(oe, ge)


@pytest.mark.parametrize("stage", [cb.LEFT, cb.MIDDLE, cb.RIGHT])
@pytest.mark.parametrize("case", ["small", "scrambled", "small_fill1", "b32_fill1"])
def test_prec_apply(handle, stage, case):
    """The fill cases give block rows and columns of more than 32 blocks and
    sparse blocks of more than 32 entries (both paths of the sweep build)."""
    fill = 1 if case.endswith("fill1") else 0
    if case.startswith("small"):
        rp, ci, v, bs = kkt("small")
    elif case == "b32_fill1":
        rp, ci, v, bs = kkt("small", block=32)
    else:
        rp, ci, v, bs = scrambled_kkt(seed=7)
    S, OF, P, F = _factor_both(handle, rp, ci, v, bs, fill_level=fill)
    b = cb.normal_vector(11, len(rp) - 1)
    xo = OF.apply(stage, b)
    xg = F.apply(stage, torch.from_numpy(b).cuda()).cpu().numpy()
    # identical operation order: exact
    assert np.array_equal(xo, xg), np.max(np.abs(xo - xg) / (np.abs(xo) + 1e-300))


@pytest.mark.parametrize("stage", [cb.LEFT, cb.MIDDLE, cb.RIGHT])
@pytest.mark.parametrize("case", ["scrambled", "small_fill1"])
def test_prec_apply_in_place(handle, stage, case):
    """b == x: LEFT gathers P' b first, MIDDLE is per row, RIGHT writes each
    block row's results at their permuted places after reading its own rows
    (pivot swaps move values inside a block row): the same bits as out of
    place, and as the oracle."""
    fill = 1 if case.endswith("fill1") else 0
    rp, ci, v, bs = kkt("small") if case.startswith("small") else scrambled_kkt(seed=7)
    S, OF, P, F = _factor_both(handle, rp, ci, v, bs, fill_level=fill)
    assert not np.array_equal(OF.export()["perm"], np.arange(len(rp) - 1)) or case != "scrambled"
    b = cb.normal_vector(13, len(rp) - 1)
    out = F.apply(stage, torch.from_numpy(b).cuda()).cpu().numpy()
    xb = torch.from_numpy(b.copy()).cuda()
    F.apply(stage, xb, xb)
    assert np.array_equal(xb.cpu().numpy(), out)
    assert np.array_equal(out, OF.apply(stage, b))


@pytest.mark.parametrize("transpose", [False, True])
def test_spmv(handle, transpose):
    rp, ci, v = random_spd_ish(500, 0.02)
    x = cb.normal_vector(5, 500)
    y0 = cb.normal_vector(6, 500)
    A = cb.CsrOperator(handle, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda(),
                       explicit_transpose=transpose)
    yg = torch.from_numpy(y0.copy()).cuda()
    A.spmv(torch.from_numpy(x).cuda(), yg, 0.5, -2.0, transpose)
    import scipy.sparse as sp

    K = sp.csr_matrix((v, ci, rp))
    ref = 0.5 * ((K.T if transpose else K) @ x) - 2.0 * y0
    assert np.allclose(yg.cpu().numpy(), ref, rtol=1e-13, atol=1e-13)


def _rows_matrix(lengths, n_cols, seed):
    rng = np.random.default_rng(seed)
    rp = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n_cols, k, replace=False)) for k in lengths] + [np.zeros(0)]).astype(np.int32)
    return rp, ci, rng.standard_normal(int(rp[-1]))


@pytest.mark.parametrize("case", ["kkt_small", "kkt_scale_rows", "ragged_empty", "rows_to_64", "long_row", "wide_rows"])
def test_spmv_bit_exact(handle, case):
    """y = alpha K x + beta y against the serial CSR loop: bit for bit where
    every row has at most 64 nonzeros and the average is at most 16 (a thread
    sums its row in column order), within rounding otherwise (warp-parallel
    sums of the long rows)."""
    if case == "kkt_small":
        rp, ci, v, _ = kkt("small")
    elif case == "kkt_scale_rows":
        rp, ci, v = cb.kkt_generate(20000, 10000, 6, 32, 1e-6, 1e6, seed=11)
    elif case == "ragged_empty":  # 1000 rows (not a multiple of the block), a third empty
        rng = np.random.default_rng(4)
        rp, ci, v = _rows_matrix(rng.integers(0, 3, 1000) * rng.integers(0, 12, 1000), 1000, 5)
    elif case == "rows_to_64":  # short rows and rows of exactly 64
        lengths = np.full(2000, 6)
        lengths[::97] = 64
        rp, ci, v = _rows_matrix(lengths, 2000, 3)
    elif case == "long_row":  # one row summed by its warp
        lengths = np.full(3000, 5)
        lengths[1234] = 2900
        rp, ci, v = _rows_matrix(lengths, 3000, 6)
    else:
        rp, ci, v = _rows_matrix(np.full(700, 40), 3000, 7)
    m = len(rp) - 1
    n_cols = int(ci.max()) + 1 if len(ci) else 1
    x = cb.normal_vector(8, max(n_cols, m))
    y0 = cb.normal_vector(9, m)
    A = cb.CsrOperator(handle, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda(),
                       ncols=len(x))
    for alpha, beta in ((1.0, 0.0), (-1.0, 1.0), (0.5, -2.0)):
        yg = torch.from_numpy(y0.copy()).cuda()
        A.spmv(torch.from_numpy(x).cuda(), yg, alpha, beta)
        ref = oracle.spmv(rp, ci, v, x, alpha, beta, y0)
        if case in ("wide_rows", "long_row"):
            assert np.allclose(yg.cpu().numpy(), ref, rtol=1e-13, atol=1e-13)
        else:
            assert np.array_equal(yg.cpu().numpy(), ref)


@pytest.mark.parametrize("case", ["kkt_small", "kkt_scale_rows", "ragged_empty", "rows_to_64", "long_row", "wide_rows"])
@pytest.mark.parametrize("precision", [cb.F64, cb.F32])
def test_spmv_sell_bit_exact(handle, case, precision):
    """The SELL-32 copy (culipx_csr_set_format): every row of at most 64
    entries is summed serially in column order, so y equals the serial CSR
    loop bit for bit at any average row length (the CSR kernel's wide rows
    are group-reduced); the one longer row keeps the warp sum.  The copy
    holds the values it was built with until culipx_csr_refresh."""
    if case == "kkt_small":
        rp, ci, v, _ = kkt("small")
    elif case == "kkt_scale_rows":
        rp, ci, v = cb.kkt_generate(20000, 10000, 6, 32, 1e-6, 1e6, seed=11)
    elif case == "ragged_empty":
        rng = np.random.default_rng(4)
        rp, ci, v = _rows_matrix(rng.integers(0, 3, 1000) * rng.integers(0, 12, 1000), 1000, 5)
    elif case == "rows_to_64":
        lengths = np.full(2000, 6)
        lengths[::97] = 64
        rp, ci, v = _rows_matrix(lengths, 2000, 3)
    elif case == "long_row":
        lengths = np.full(3000, 5)
        lengths[1234] = 2900
        rp, ci, v = _rows_matrix(lengths, 3000, 6)
    else:
        rp, ci, v = _rows_matrix(np.full(700, 40), 3000, 7)
    m = len(rp) - 1
    n_cols = int(ci.max()) + 1 if len(ci) else 1
    dt = np.float64 if precision == cb.F64 else np.float32
    x = cb.normal_vector(8, max(n_cols, m)).astype(dt)
    y0 = cb.normal_vector(9, m).astype(dt)
    vt = torch.from_numpy(v.astype(dt)).cuda()
    A = cb.CsrOperator(handle, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), vt, ncols=len(x))
    A.set_format(cb.FMT_SELL)

    def check(vals):
        for alpha, beta in ((1.0, 0.0), (-1.0, 1.0), (0.5, -2.0)):
            yg = torch.from_numpy(y0.copy()).cuda()
            A.spmv(torch.from_numpy(x).cuda(), yg, alpha, beta)
            y = yg.cpu().numpy()
            if precision == cb.F64:
                ref = oracle.spmv(rp, ci, vals, x, alpha, beta, y0)
                if case == "long_row":
                    assert np.allclose(y, ref, rtol=1e-13, atol=1e-13)
                else:
                    assert np.array_equal(y, ref)
            else:
                A.set_format(cb.FMT_CSR)
                yc = torch.from_numpy(y0.copy()).cuda()
                A.spmv(torch.from_numpy(x).cuda(), yc, alpha, beta)
                A.set_format(cb.FMT_SELL)
                if case in ("kkt_small", "kkt_scale_rows", "ragged_empty", "rows_to_64"):
                    assert np.array_equal(y, yc.cpu().numpy())
                else:
                    assert np.allclose(y, yc.cpu().numpy(), rtol=1e-4, atol=1e-4)

    check(v.astype(dt).astype(np.float64))
    if precision == cb.F64:
        vt.mul_(-3.0)
        check(v)  # the copy still holds the old values
        A.refresh()
        check(-3.0 * v)


def test_sqmr_small_kkt(handle):
    rp, ci, v, bs = kkt("small")
    S, OF, P, F = _factor_both(handle, rp, ci, v, bs)
    b = cb.normal_vector(cb.SEED + 1, len(rp) - 1)
    xo, reso, ito = oracle.sqmr(rp, ci, v, b, OF, 1e-8, 1000)
    A = cb.CsrOperator(handle, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    xg = torch.zeros(len(rp) - 1, dtype=torch.float64, device="cuda")
    res, its, st = cb.sqmr_solve(handle, A, F, torch.from_numpy(b).cuda(), xg, 1e-8, 1000)
    xg = xg.cpu().numpy()
    # same recurrence and check protocol; reductions differ only in summation order
    assert abs(its - ito) <= 4
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) < 1e-6
    r = b - oracle.spmv(rp, ci, v, xg)
    ro = b - oracle.spmv(rp, ci, v, xo)
    assert np.linalg.norm(r) <= 2 * np.linalg.norm(ro) + 1e-12 * np.linalg.norm(b)


def _csr_op(handle, rp, ci, v):
    return cb.CsrOperator(handle, torch.from_numpy(np.ascontiguousarray(rp, np.int32)).cuda(),
                          torch.from_numpy(np.ascontiguousarray(ci, np.int32)).cuda(),
                          torch.from_numpy(np.ascontiguousarray(v, np.float64)).cuda())


@pytest.mark.parametrize("fill_level", [0, 1])
def test_sqmr_deep_levels(handle, fill_level):
    """Random symmetric indefinite matrix, random blocking: many levels in the
    persistent solver's sweeps."""
    from problems import random_blocking

    rp, ci, v = random_spd_ish(900, 0.01, seed=12)
    bs = random_blocking(900, np.random.default_rng(3), 2, 20)
    S, OF, P, F = _factor_both(handle, rp, ci, v, bs, fill_level=fill_level)
    assert P.info()["num_levels"] > 5
    b = cb.normal_vector(21, len(rp) - 1)
    xo, reso, ito = oracle.sqmr(rp, ci, v, b, OF, 1e-10, 500)
    A = _csr_op(handle, rp, ci, v)
    xg = torch.zeros(len(rp) - 1, dtype=torch.float64, device="cuda")
    res, its, st = cb.sqmr_solve(handle, A, F, torch.from_numpy(b).cuda(), xg, 1e-10, 500)
    xg = xg.cpu().numpy()
    assert abs(its - ito) <= 4
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) < 1e-6
    import scipy.sparse as sp

    K = sp.csr_matrix((v, ci, rp))
    assert np.linalg.norm(b - K @ xg) / np.linalg.norm(b) < 1e-6


def test_sqmr_reference_fixture_unpreconditioned(handle):
    """tests/la/test_sqmr.cc small_D: SQMR without preconditioner, term_tol 1e-10,
    ||b - A x|| <= 1e-5 ||b||, iterations <= n."""
    import os

    d = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sqmr_small.npz"))
    rp, ci, v = d["A_rowptr"], d["A_colidx"], d["A_val"]
    n = len(rp) - 1
    import scipy.sparse as sp

    Kh = sp.csr_matrix((v, ci, rp), shape=(n, n))
    b = Kh @ np.ones(n)
    A = _csr_op(handle, rp, ci, v)
    xg = torch.zeros(n, dtype=torch.float64, device="cuda")
    res, its, st = cb.sqmr_solve(handle, A, None, torch.from_numpy(b).cuda(), xg, 1e-10, n)
    x = xg.cpu().numpy()
    assert np.linalg.norm(b - Kh @ x) <= 1e-5 * np.linalg.norm(b)
    assert its <= n
    xo, reso, ito = oracle.sqmr(rp, ci, v, b, None, 1e-10, n)
    assert abs(its - ito) <= 4


@pytest.mark.parametrize("precision", [cb.F64, cb.F32])
@pytest.mark.parametrize("nrhs", [1, 2, 3, 4, 6])
def test_sqmr_multi_rhs(handle, precision, nrhs):
    """Several right-hand sides in one launch: each follows its own SQMR
    recurrence and stopping test, so it matches its single-RHS solve up to
    summation order, and its x stays final once it stops."""
    rp, ci, v, bs = kkt("small")
    n = len(rp) - 1
    P = cb.Pattern(handle, rp, ci, bs, 0, 1.0, precision)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v.astype(np.float32 if precision == cb.F32 else np.float64)).cuda())
    A = _csr_op(handle, rp, ci, v)
    rng = np.random.default_rng(77 + nrhs)
    B = rng.standard_normal((nrhs, n))
    B[-1] *= 1e-3  # a small right-hand side converges at its own iteration
    X = torch.full((nrhs, n), 7.0, dtype=torch.float64, device="cuda")
    res, its, st = cb.sqmr_solve_multi(handle, A, F, torch.from_numpy(B).cuda(), X, 1e-8, 1000)
    import scipy.sparse as sp

    K = sp.csr_matrix((v, ci, rp))
    X = X.cpu().numpy()
    for r in range(nrhs):
        x1 = torch.zeros(n, dtype=torch.float64, device="cuda")
        r1, i1, s1 = cb.sqmr_solve(handle, A, F, torch.from_numpy(B[r]).cuda(), x1, 1e-8, 1000)
        x1 = x1.cpu().numpy()
        assert st[r] == s1 == capi.OK
        assert abs(int(its[r]) - i1) <= 4
        assert np.linalg.norm(X[r] - x1) / np.linalg.norm(x1) < 1e-6
        rel = np.linalg.norm(B[r] - K @ X[r]) / np.linalg.norm(B[r])
        rel1 = np.linalg.norm(B[r] - K @ x1) / np.linalg.norm(B[r])
        assert rel <= 2 * rel1 + 1e-12
    if precision == cb.F64:
        xo, _, ito = oracle.sqmr(rp, ci, v, B[0], _oracle_factor(rp, ci, v, bs), 1e-8, 1000)
        assert abs(int(its[0]) - ito) <= 4


@pytest.mark.parametrize("nrhs", [1, 3, 5])
def test_sqmr_refine_multi(handle, nrhs):
    """FP32 factor, FP64 refinement, several right-hand sides: every column
    reaches the tolerance in about the corrections its single refinement
    takes, and columns of very different scale stop independently."""
    rp, ci, v, bs = kkt("small")
    n = len(rp) - 1
    P = cb.Pattern(handle, rp, ci, bs, 0, 1.0, cb.F32)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v.astype(np.float32)).cuda())
    A = _csr_op(handle, rp, ci, v)
    rng = np.random.default_rng(5 + nrhs)
    B = rng.standard_normal((nrhs, n)) * (10.0 ** np.arange(nrhs))[:, None]
    X = torch.zeros((nrhs, n), dtype=torch.float64, device="cuda")
    rel, its, steps, st = cb.sqmr_refine_multi(handle, A, F, torch.from_numpy(B).cuda(), X, 1e-10, 1e-6, 1000, 20)
    import scipy.sparse as sp

    K = sp.csr_matrix((v, ci, rp))
    X = X.cpu().numpy()
    for r in range(nrhs):
        assert st[r] == capi.OK and rel[r] <= 1e-10
        true = np.linalg.norm(B[r] - K @ X[r]) / np.linalg.norm(B[r])
        assert abs(true - rel[r]) <= 1e-3 * rel[r] + 1e-15
        x1 = torch.zeros(n, dtype=torch.float64, device="cuda")
        r1, i1, s1, st1 = cb.sqmr_refine(handle, A, F, torch.from_numpy(B[r]).cuda(), x1, 1e-10, 1e-6, 1000, 20)
        assert st1 == capi.OK and abs(int(steps[r]) - s1) <= 1


def _oracle_factor(rp, ci, v, bs):
    return oracle.Sym(rp, ci, bs, 0, 1.0).factor(v)


def test_sqmr_fp32_factor_mixed(handle):
    """FP32 factor and applies, FP64 recurrence: converges on the small KKT."""
    rp, ci, v, bs = kkt("small")
    P = cb.Pattern(handle, rp, ci, bs, 0, 1.0, cb.F32)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v.astype(np.float32)).cuda())
    b = cb.normal_vector(cb.SEED + 1, len(rp) - 1)
    A = _csr_op(handle, rp, ci, v)
    xg = torch.zeros(len(rp) - 1, dtype=torch.float64, device="cuda")
    res, its, st = cb.sqmr_solve(handle, A, F, torch.from_numpy(b).cuda(), xg, 1e-8, 1000)
    import scipy.sparse as sp

    K = sp.csr_matrix((v, ci, rp))
    assert np.linalg.norm(b - K @ xg.cpu().numpy()) / np.linalg.norm(b) < 1e-4


@pytest.mark.parametrize("stage", [cb.LEFT, cb.RIGHT])
@pytest.mark.parametrize("sweeps", [0, 1, 3, "levels"])
def test_prec_apply_jacobi(handle, stage, sweeps):
    """SOLVE_JACOBI (set_solve_algorithm): block-Jacobi sweeps from x = 0,
    bit-exact against the oracle; with as many sweeps as levels it is the
    exact solve."""
    rp, ci, v, bs = scrambled_kkt(seed=8)
    S, OF, P, F = _factor_both(handle, rp, ci, v, bs)
    nl = P.info()["num_levels"]
    sw = nl if sweeps == "levels" else sweeps
    F.set_solve_algorithm(cb.SOLVE_JACOBI, sw)
    b = cb.normal_vector(13, len(rp) - 1)
    xo = OF.apply(stage, b, jacobi_sweeps=sw) if sw > 0 else np.zeros_like(b)
    xg = F.apply(stage, torch.from_numpy(b).cuda()).cpu().numpy()
    assert np.array_equal(xo, xg)
    if sweeps == "levels":
        assert np.array_equal(xg, OF.apply(stage, b))
    F.set_solve_algorithm(cb.SOLVE_BLOCK, 0)
    assert np.array_equal(F.apply(stage, torch.from_numpy(b).cuda()).cpu().numpy(), OF.apply(stage, b))


def test_sqmr_jacobi(handle):
    """SQMR with the SOLVE_JACOBI preconditioner (2 sweeps) against the oracle."""
    rp, ci, v, bs = kkt("small")
    S, OF, P, F = _factor_both(handle, rp, ci, v, bs)
    F.set_solve_algorithm(cb.SOLVE_JACOBI, 2)
    b = cb.normal_vector(cb.SEED + 1, len(rp) - 1)
    xo, reso, ito = oracle.sqmr(rp, ci, v, b, OF, 1e-8, 1000, jacobi_sweeps=2)
    A = _csr_op(handle, rp, ci, v)
    xg = torch.zeros(len(rp) - 1, dtype=torch.float64, device="cuda")
    res, its, st = cb.sqmr_solve(handle, A, F, torch.from_numpy(b).cuda(), xg, 1e-8, 1000)
    xg = xg.cpu().numpy()
    assert abs(its - ito) <= 4
    assert np.linalg.norm(xg - xo) / np.linalg.norm(xo) < 1e-6


@pytest.mark.parametrize("precision", [cb.F32, cb.F64])
def test_sqmr_refine_small(handle, precision):
    """FP64 iterative refinement around SQMR reaches a true relative residual
    the single FP32-factor solve cannot (1e-10); the returned relres is the
    true one, and the solution agrees with the FP64 oracle's SQMR solve."""
    rp, ci, v, bs = kkt("small")
    P = cb.Pattern(handle, rp, ci, bs, 0, 1.0, precision)
    F = cb.Factor(P)
    dt = np.float32 if precision == cb.F32 else np.float64
    F.compute(torch.from_numpy(v.astype(dt)).cuda())
    b = cb.normal_vector(cb.SEED + 1, len(rp) - 1)
    A = _csr_op(handle, rp, ci, v)
    xg = torch.zeros(len(rp) - 1, dtype=torch.float64, device="cuda")
    rel, its, steps, st = cb.sqmr_refine(handle, A, F, torch.from_numpy(b).cuda(), xg, 1e-10, 1e-6, 1000, 20)
    import scipy.sparse as sp

    K = sp.csr_matrix((v, ci, rp))
    x = xg.cpu().numpy()
    true_rel = np.linalg.norm(b - K @ x) / np.linalg.norm(b)
    assert st == capi.OK and rel <= 1e-10 and steps >= 1
    assert abs(true_rel - rel) <= 1e-3 * rel + 1e-15
    S = oracle.Sym(rp, ci, bs, 0, 1.0)
    xo, _, _ = oracle.sqmr(rp, ci, v, b, S.factor(v), 1e-12, 2000)
    assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-4
