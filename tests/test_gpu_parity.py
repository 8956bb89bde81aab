"""GPU parity: the sm_100a path through the C ABI against the CPU oracle.

Factor, D, pivots and permutation are compared exactly (the kernels and the
oracle spell out the same roundings); preconditioner applies, SpMV and SQMR
with stated tolerances.
"""
import numpy as np
import pytest

import culip_b200 as cb
import oracle
from problems import kkt, random_spd_ish, scrambled_kkt

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def handle():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return cb.Handle(0)


def _factor_both(handle, rp, ci, v, bs, fill_level=0, pivot=cb.PIV_BK, precision=cb.F64, is_piv=None):
    dt = np.float64 if precision == cb.F64 else np.float32
    S = oracle.Sym(rp, ci, bs, fill_level, 1.0, dtype=dt)
    OF = S.factor(v.astype(dt), is_piv=is_piv, pivot=pivot)
    P = cb.Pattern(handle, rp, ci, bs, fill_level, 1.0, precision)
    F = cb.Factor(P)
    tv = torch.from_numpy(v.astype(dt)).cuda()
    F.compute(tv, is_piv=is_piv, pivot=pivot)
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
@pytest.mark.parametrize("case", ["small", "scrambled"])
def test_prec_apply(handle, stage, case):
    if case == "small":
        rp, ci, v, bs = kkt("small")
    else:
        rp, ci, v, bs = scrambled_kkt(seed=7)
    S, OF, P, F = _factor_both(handle, rp, ci, v, bs)
    b = cb.normal_vector(11, len(rp) - 1)
    xo = OF.apply(stage, b)
    xg = F.apply(stage, torch.from_numpy(b).cuda()).cpu().numpy()
    # identical operation order: exact
    assert np.array_equal(xo, xg), np.max(np.abs(xo - xg) / (np.abs(xo) + 1e-300))


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
