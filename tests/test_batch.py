"""Batched solves: independent KKT systems of uneven size stored as one
block-diagonal union (one pattern, one factor) and solved in one launch, one
CTA per system.  Each system's result must be the same alone and in the mix
(bit for bit) and agree with the oracle's SQMR on that system alone."""
import numpy as np
import pytest
import scipy.sparse as sp

import culip_b200 as cb
from culip_b200 import _capi as capi
import oracle
from problems import scrambled_kkt


def _systems(count=6, seed=100):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.integers(200, 1500))
        m = n // 2
        rp, ci, v = cb.kkt_generate(n, m, int(rng.integers(4, 9)), 16, 1e-3, 1e3, seed=cb.SEED + 1000 * 4 + k)
        bs = cb.kkt_blocking(n, m, 16)
        out.append((rp, ci, v, bs))
    return out


def test_union_systems_is_block_diagonal():
    syst = _systems(3)
    rp, ci, v, bs, off = cb.union_systems(syst)
    U = sp.csr_matrix((v, ci, rp)).toarray()
    B = sp.block_diag([sp.csr_matrix((s[2], s[1], s[0])) for s in syst]).toarray()
    assert np.array_equal(U, B)
    assert off[0] == 0 and off[-1] == len(rp) - 1
    assert set(off[:-1]).issubset(set(bs))


def _rhs(syst, ids):
    return [cb.normal_vector(cb.SEED + 7 + k, len(s[0]) - 1) for k, s in zip(ids, syst)]


def _solve_batch(handle, syst, precision=cb.F64, tol=1e-8, max_it=1000, rhs=None):
    import torch

    rp, ci, v, bs, off = cb.union_systems(syst)
    P = cb.Pattern(handle, rp, ci, bs, 0, 1.0, precision, system_row_offsets=off)
    F = cb.Factor(P)
    dt = np.float64 if precision == cb.F64 else np.float32
    F.compute(torch.from_numpy(v.astype(dt)).cuda())
    A = cb.CsrOperator(handle, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    bvec = np.concatenate(rhs if rhs is not None else _rhs(syst, range(len(syst))))
    x = torch.zeros(len(rp) - 1, dtype=torch.float64, device="cuda")
    B = cb.Batch(P, off)
    res, its, st = cb.batch_sqmr_solve(B, A, F, torch.from_numpy(bvec).cuda(), x, tol, max_it)
    # natural-order KKT systems at level-0 fill draw no extra capacity, so the
    # union factor equals the separate factors
    assert F.info()["granted_blocks"] == 0
    return x.cpu().numpy(), res, its, st, off, bvec


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [cb.F64, cb.F32])
def test_batch_same_alone_and_in_the_mix(precision):
    h = cb.Handle(0)
    syst = _systems(6)
    rhs = _rhs(syst, range(6))
    x, res, its, st, off, bvec = _solve_batch(h, syst, precision, rhs=rhs)
    assert np.all(st != capi.BREAKDOWN)
    for k in (0, 3, 5):
        xk, resk, itsk, stk, offk, _ = _solve_batch(h, [syst[k]], precision, rhs=[rhs[k]])
        # the mix holds the same right-hand side for system k
        assert np.array_equal(x[off[k]:off[k + 1]], xk)
        assert its[k] == itsk[0] and res[k] == resk[0] and st[k] == stk[0]
    # a different mix (reversed order) gives the same per-system results
    xr, resr, itsr, _, offr, _ = _solve_batch(h, syst[::-1], precision, rhs=rhs[::-1])
    for k in range(6):
        j = 5 - k
        assert its[k] == itsr[j] and res[k] == resr[j]
        assert np.array_equal(x[off[k]:off[k + 1]], xr[offr[j]:offr[j + 1]])


@pytest.mark.gpu
def test_batch_matches_oracle_per_system():
    h = cb.Handle(0)
    syst = _systems(6, seed=7)
    x, res, its, st, off, bvec = _solve_batch(h, syst)
    for k, (rp, ci, v, bs) in enumerate(syst):
        b = bvec[off[k]:off[k + 1]]
        S = oracle.Sym(rp, ci, bs, 0, 1.0)
        xo, reso, ito = oracle.sqmr(rp, ci, v, b, S.factor(v), 1e-8, 1000)
        assert abs(int(its[k]) - ito) <= 4, (k, its[k], ito)
        xk = x[off[k]:off[k + 1]]
        # both solves stop at tol 1e-8 on the quasi-residual; their iterates
        # differ by rounding amplified by the system's conditioning
        assert np.linalg.norm(xk - xo) / np.linalg.norm(xo) < 1e-4
        K = sp.csr_matrix((v, ci, rp))
        ro = np.linalg.norm(b - K @ xo)
        # the quasi-residual test stops both at tol; their true residuals are
        # rounding-sensitive at this level (a factor of a few either way)
        assert np.linalg.norm(b - K @ xk) <= 10 * ro + 1e-12 * np.linalg.norm(b)


@pytest.mark.gpu
def test_batch_rejects_coupled_or_split_systems():
    import torch

    h = cb.Handle(0)
    syst = _systems(2)
    rp, ci, v, bs, off = cb.union_systems(syst)
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F64)
    with pytest.raises(cb.CulipxError):
        cb.Batch(P, [0, off[1] + 1, off[2]])  # splits a block row
    with pytest.raises(cb.CulipxError):
        cb.Batch(P, [0, off[2] + 1])  # does not end at n
    # a coupling entry between the two systems
    K = sp.csr_matrix((v, ci, rp)).tolil()
    K[0, off[1]] = 1.0
    K[off[1], 0] = 1.0
    K = K.tocsr()
    K.sort_indices()
    P2 = cb.Pattern(h, K.indptr.astype(np.int32), K.indices.astype(np.int32), bs, 0, 1.0, cb.F64)
    with pytest.raises(cb.CulipxError):
        cb.Batch(P2, off)
    del torch


@pytest.mark.gpu
def test_batch_union_shares_the_leftover_pool():
    """A scrambled system whose off-diagonal blocks overflow their fill cap
    draws extra capacity from the factorization's single leftover pool (one
    pool per factorization, as in the reference); factor_info reports it, so
    a caller can tell when a union factor may differ from separate factors.
    (Scrambled KKT systems are too sensitive for an SQMR comparison: even
    two exact-arithmetic-equivalent solves differ by hundreds of iterations.)"""
    import torch

    h = cb.Handle(0)
    syst = _systems(2, seed=3) + [scrambled_kkt(seed=9)]
    rp, ci, v, bs, off = cb.union_systems(syst)
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F64)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v).cuda())
    assert F.info()["granted_blocks"] > 0
    r2, c2, v2, b2 = syst[2]
    P2 = cb.Pattern(h, r2, c2, b2, 0, 1.0, cb.F64)
    F2 = cb.Factor(P2)
    F2.compute(torch.from_numpy(v2).cuda())
    assert F2.info()["granted_blocks"] > 0
    for s in syst[:2]:
        Ps = cb.Pattern(h, s[0], s[1], s[3], 0, 1.0, cb.F64)
        Fs = cb.Factor(Ps)
        Fs.compute(torch.from_numpy(s[2]).cuda())
        assert Fs.info()["granted_blocks"] == 0


@pytest.mark.gpu
def test_batch_refine_fp32_reaches_tol():
    """FP32 union factor, batched FP64 refinement: every system reaches a true
    relative residual of 1e-10, checked on the host per system."""
    import torch

    h = cb.Handle(0)
    syst = _systems(6, seed=21)
    rp, ci, v, bs, off = cb.union_systems(syst)
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F32, system_row_offsets=off)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v.astype(np.float32)).cuda())
    A = cb.CsrOperator(h, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    b = np.concatenate(_rhs(syst, range(6)))
    x = torch.zeros(len(rp) - 1, dtype=torch.float64, device="cuda")
    rel, its, steps, st = cb.batch_sqmr_refine(cb.Batch(P, off), A, F, torch.from_numpy(b).cuda(), x, 1e-10, 1e-6,
                                               1000, 20)
    xs = x.cpu().numpy()
    for k, (srp, sci, sv, sbs) in enumerate(syst):
        K = sp.csr_matrix((sv, sci, srp))
        bk = b[off[k]:off[k + 1]]
        true_rel = np.linalg.norm(bk - K @ xs[off[k]:off[k + 1]]) / np.linalg.norm(bk)
        assert st[k] == capi.OK and rel[k] <= 1e-10 and steps[k] >= 1
        assert abs(true_rel - rel[k]) <= 1e-3 * rel[k] + 1e-15


def test_union_analysis_formats_equal_separate_analyses():
    """With system boundaries, the union's block formats and fill caps are the
    concatenation of the separate analyses' (host-only handle, no GPU)."""
    import ctypes

    class HostHandle:
        def __init__(self):
            self._h = ctypes.c_void_p()
            capi.call("culipx_handle_create", ctypes.byref(self._h), -1, None)

    hh = HostHandle()
    syst = _systems(4, seed=5)
    rp, ci, v, bs, off = cb.union_systems(syst)
    U = cb.Pattern(hh, rp, ci, bs, 0, 1.0, cb.F32, system_row_offsets=off).export()
    fmts, mx = [], []
    for s in syst:
        E = cb.Pattern(hh, s[0], s[1], s[3], 0, 1.0, cb.F32).export()
        fmts.append(E["fmt"])
        mx.append(E["max_nnz"])
    assert np.array_equal(U["fmt"], np.concatenate(fmts))
    assert np.array_equal(U["max_nnz"], np.concatenate(mx))
    with pytest.raises(cb.CulipxError):
        cb.Pattern(hh, rp, ci, bs, 0, 1.0, cb.F32, system_row_offsets=[0, off[1] + 1, off[-1]])
    capi.load().culipx_handle_destroy(hh._h)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [cb.F64, cb.F32])
def test_batch_factor_solve_graph_replays_bit_for_bit(precision):
    """culipx_batch_factor_solve_graph: the factorization of the union and the
    batched solve as one graph launch.  The capturing call and two replays
    (the second after the values changed) each equal an ordinary factor +
    batch_sqmr_solve of the same values, bit for bit."""
    import torch

    handle = cb.Handle(0)
    syst = _systems(5, seed=321)
    rp, ci, v, bs, off = cb.union_systems(syst)
    dt = torch.float64 if precision == cb.F64 else torch.float32
    P = cb.Pattern(handle, rp, ci, bs, 0, 1.0, precision, system_row_offsets=off)
    F, F2 = cb.Factor(P), cb.Factor(P)
    B = cb.Batch(P, off)
    d_v = torch.from_numpy(v).cuda()
    d_vals = d_v.to(dt)
    A = cb.CsrOperator(handle, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), d_v)
    b = torch.from_numpy(np.concatenate(_rhs(syst, range(len(syst))))).cuda()
    x = torch.zeros_like(b)
    x2 = torch.zeros_like(b)
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    diag = torch.from_numpy(np.nonzero(rows == ci)[0]).cuda()
    for call in range(3):
        if call == 2:  # new values behind the same buffers: the replay must pick them up
            d_v[diag] *= 1.5
            d_vals.copy_(d_v.to(dt))
        res, its, st = cb.batch_factor_solve_graph(B, A, F, d_vals, b, x, 1e-8, 300)
        F2.compute(d_vals.clone())
        res2, its2, st2 = cb.batch_sqmr_solve(B, A, F2, b, x2, 1e-8, 300)
        assert np.array_equal(its, its2) and np.array_equal(st, st2) and np.array_equal(res, res2), call
        assert torch.equal(x, x2), call
        for k in ("val", "tri", "perm"):
            assert np.array_equal(F.export()[k], F2.export()[k]), (call, k)
