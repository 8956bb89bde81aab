"""The request server and the many-factor batched solve: every result is the
same alone and in the mix (bit for bit), agrees with the oracle, and the
memory budget bounds what runs at once without starving any request."""
import numpy as np
import pytest

import culip_b200 as cb
from culip_b200 import _capi as capi
import oracle

pytestmark = pytest.mark.gpu


def _patterns(count=3, seed=40):
    rng = np.random.default_rng(seed)
    pats = []
    for k in range(count):
        n = int(rng.integers(300, 1200))
        m = n // 2
        rp, ci, v = cb.kkt_generate(n, m, 6, 16, 1e-3, 1e3, seed=cb.SEED + 5000 + k)
        pats.append((rp, ci, v, cb.kkt_blocking(n, m, 16)))
    return pats


def _ipm_values(rp, ci, v, n_h, rng):
    """The next IPM iteration's values: H scaled by 10^U(-1, 1), clipped."""
    out = v.copy()
    rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
    diag = (rows == ci) & (rows < n_h)
    h = out[diag] - 1e-8
    out[diag] = np.clip(h * 10.0 ** rng.uniform(-1, 1, diag.sum()), 1e-8, 1e8) + 1e-8
    return out


def _requests(pats, count, seed):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        p = int(rng.integers(0, len(pats)))
        rp, ci, v, bs = pats[p]
        n_h = (len(rp) - 1) * 2 // 3  # H rows: n of N = n + n // 2
        vals = _ipm_values(rp, ci, v, n_h, rng)
        nrhs = int(rng.integers(1, 4))
        b = rng.standard_normal((len(rp) - 1, nrhs))
        reqs.append((p, vals, b))
    return reqs


def _serve(pats, reqs, slots=2, max_batch=4, budget=0, large_rows=None, precision=cb.F64):
    s = cb.Server(0, budget, slots, max_batch, 1e-8, 1000)
    if large_rows is not None:
        s.set_large_rows(large_rows)
    pids = [s.add_pattern(rp, ci, bs, precision) for rp, ci, v, bs in pats]
    ids = [s.submit(pids[p], vals, b) for p, vals, b in reqs]
    done = 0
    while done < len(ids):
        done += s.progress(wait=True)
    out = [s.result(i) for i in ids]
    return out, s


def test_server_same_alone_and_in_the_mix():
    pats = _patterns()
    reqs = _requests(pats, 10, seed=1)
    mixed, s = _serve(pats, reqs)
    st = s.stats()
    assert st["done"] == 10 and st["queued"] == 0 and st["running"] == 0 and st["batches"] >= 3
    for k in (0, 4, 9):
        alone, _ = _serve(pats, [reqs[k]], slots=1, max_batch=1)
        x, its, status, lat = mixed[k]
        xa, itsa, sta, lata = alone[0]
        assert np.array_equal(x, xa) and np.array_equal(its, itsa) and np.array_equal(status, sta)
        assert lat > 0
    # agreement with the oracle on one request
    p, vals, b = reqs[3]
    rp, ci, v, bs = pats[p]
    S = oracle.Sym(rp, ci, bs, 0, 1.0)
    F = S.factor(vals)
    x, its, status, lat = mixed[3]
    for r in range(b.shape[1]):
        xo, _, ito = oracle.sqmr(rp, ci, vals, b[:, r], F, 1e-8, 1000)
        # hundreds of iterations: the summation orders' rounding shifts the count a little
        assert abs(int(its[r]) - ito) <= max(4, 0.05 * ito)
        assert np.linalg.norm(x[:, r] - xo) / np.linalg.norm(xo) < 1e-4


def test_server_large_requests_whole_gpu_path():
    """Patterns at or above the large-row threshold are solved by the
    whole-GPU solver in batches of their own that run alone; results are the
    same alone and in the mix, and agree with the oracle."""
    pats = []
    for k, n in enumerate((400, 900, 1100)):  # N = 600 (small), 1350, 1650 (large)
        rp, ci, v = cb.kkt_generate(n, n // 2, 6, 16, 1e-3, 1e3, seed=cb.SEED + 5100 + k)
        pats.append((rp, ci, v, cb.kkt_blocking(n, n // 2, 16)))
    reqs = _requests(pats, 9, seed=4)
    mixed, s = _serve(pats, reqs, slots=2, max_batch=4, large_rows=1000)
    st = s.stats()
    assert st["done"] == 9 and st["large_batches"] >= 1 and st["batches"] > st["large_batches"]
    for k in range(9):
        alone, _ = _serve(pats, [reqs[k]], slots=1, max_batch=1, large_rows=1000)
        assert np.array_equal(mixed[k][0], alone[0][0]) and np.array_equal(mixed[k][1], alone[0][1])
    # a large request against the oracle
    k = next(i for i, (p, _, _) in enumerate(reqs) if len(pats[p][0]) - 1 >= 1000)
    p, vals, b = reqs[k]
    rp, ci, v, bs = pats[p]
    F = oracle.Sym(rp, ci, bs, 0, 1.0).factor(vals)
    x, its, status, lat = mixed[k]
    for r in range(b.shape[1]):
        xo, _, ito = oracle.sqmr(rp, ci, vals, b[:, r], F, 1e-8, 1000)
        assert abs(int(its[r]) - ito) <= max(4, 0.05 * ito)
        assert np.linalg.norm(x[:, r] - xo) / np.linalg.norm(xo) < 1e-4


@pytest.mark.parametrize("large_rows", [None, 1000])
def test_server_fp32_factors(large_rows):
    """FP32 factors (FP64 SQMR): both solver classes, the same alone and in
    the mix; the SQMR stopping test (tol 1e-8 on the quasi-residual, which an
    FP32 preconditioner bounds) leaves a true residual of about 1e-4."""
    import scipy.sparse as sp

    pats = []
    for k, n in enumerate((400, 900)):  # N = 600, 1350
        rp, ci, v = cb.kkt_generate(n, n // 2, 6, 16, 1e-3, 1e3, seed=cb.SEED + 5200 + k)
        pats.append((rp, ci, v, cb.kkt_blocking(n, n // 2, 16)))
    reqs = _requests(pats, 6, seed=5)
    mixed, s = _serve(pats, reqs, large_rows=large_rows, precision=cb.F32)
    assert s.stats()["done"] == 6
    for k in (0, 5):
        alone, _ = _serve(pats, [reqs[k]], slots=1, max_batch=1, large_rows=large_rows, precision=cb.F32)
        assert np.array_equal(mixed[k][0], alone[0][0])
    for (p, vals, b), (x, its, status, lat) in zip(reqs, mixed):
        rp, ci, v, bs = pats[p]
        K = sp.csr_matrix((vals, ci, rp))
        for r in range(b.shape[1]):
            assert status[r] == capi.OK
            assert np.linalg.norm(b[:, r] - K @ x[:, r]) / np.linalg.norm(b[:, r]) < 5e-3


def test_server_grouped_right_hand_sides():
    """A batch of more than 4 x 296 right-hand sides is solved four (then two,
    one) right-hand sides per CTA: every request's result agrees with the
    same request served alone (one right-hand side per CTA)."""
    n = 300
    rp, ci, v = cb.kkt_generate(n, n // 2, 6, 16, 1e-3, 1e3, seed=cb.SEED + 5300)
    pats = [(rp, ci, v, cb.kkt_blocking(n, n // 2, 16))]
    rng = np.random.default_rng(6)
    reqs = []
    for i in range(160):
        vals = _ipm_values(rp, ci, v, n, rng)
        reqs.append((0, vals, rng.standard_normal((len(rp) - 1, 8 if i % 10 else 7))))
    mixed, s = _serve(pats, reqs, slots=1, max_batch=512)
    assert s.stats()["batches"] == 1  # one batch of 1264 right-hand sides
    for k in (0, 9, 10, 159):
        alone, _ = _serve(pats, [reqs[k]], slots=1, max_batch=1)
        assert np.array_equal(mixed[k][1], alone[0][1])
        assert np.allclose(mixed[k][0], alone[0][0], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("large_rows", [None, 1000])
def test_server_fp32_refined(large_rows):
    """FP32 factors with FP64 refinement: every right-hand side ends with a
    true relative residual at most tol (1e-8), computed here in FP64; the
    same alone and in the mix."""
    import scipy.sparse as sp

    pats = []
    for k, n in enumerate((400, 900)):  # N = 600, 1350
        rp, ci, v = cb.kkt_generate(n, n // 2, 6, 16, 1e-3, 1e3, seed=cb.SEED + 5400 + k)
        pats.append((rp, ci, v, cb.kkt_blocking(n, n // 2, 16)))
    reqs = _requests(pats, 6, seed=7)

    def serve(rq, slots, mb):
        s = cb.Server(0, 0, slots, mb, 1e-8, 1000)
        if large_rows is not None:
            s.set_large_rows(large_rows)
        s.set_refine(10, 1e-6)
        pids = [s.add_pattern(rp, ci, bs, cb.F32) for rp, ci, v, bs in pats]
        ids = [s.submit(pids[p], vals, b) for p, vals, b in rq]
        done = 0
        while done < len(ids):
            done += s.progress(wait=True)
        return [s.result(i) for i in ids]

    mixed = serve(reqs, 2, 4)
    for (p, vals, b), (x, its, status, lat) in zip(reqs, mixed):
        rp, ci, v, bs = pats[p]
        K = sp.csr_matrix((vals, ci, rp))
        for r in range(b.shape[1]):
            assert status[r] == capi.OK
            assert np.linalg.norm(b[:, r] - K @ x[:, r]) / np.linalg.norm(b[:, r]) <= 1.0001e-8
    alone = serve([reqs[2]], 1, 1)
    assert np.array_equal(alone[0][0], mixed[2][0]) and np.array_equal(alone[0][1], mixed[2][1])


def test_server_memory_budget_serializes_but_completes():
    pats = _patterns(2, seed=41)
    reqs = _requests(pats, 6, seed=2)
    big, _ = _serve(pats, reqs)
    # a budget that holds the patterns and little more: one request at a time
    s0 = cb.Server(0, 0, 1, 1, 1e-8, 1000)
    for rp, ci, v, bs in pats:
        s0.add_pattern(rp, ci, bs)
    budget = s0.stats()["held_bytes"] + 1_000_000
    small, s = _serve(pats, reqs, slots=2, max_batch=8, budget=budget)
    assert s.stats()["batches"] == len(reqs)
    for a, b in zip(big, small):
        assert np.array_equal(a[0], b[0])


def test_solve_many_matches_alone():
    import torch

    h = cb.Handle(0)
    pats = _patterns(4, seed=42)
    As, Fs, bs, xs, keep = [], [], [], [], []
    for rp, ci, v, bl in pats:
        P = cb.Pattern(h, rp, ci, bl, 0, 1.0, cb.F64)
        F = cb.Factor(P)
        F.compute(torch.from_numpy(v).cuda())
        A = cb.CsrOperator(h, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
        b = torch.from_numpy(cb.normal_vector(cb.SEED + 9, len(rp) - 1)).cuda()
        keep.append(P)
        As.append(A)
        Fs.append(F)
        bs.append(b)
        xs.append(torch.zeros_like(b))
    res, its, st = cb.sqmr_solve_many(h, As, Fs, bs, xs, 1e-8, 1000)
    for k in range(4):
        x1 = torch.zeros_like(bs[k])
        r1, i1, s1 = cb.sqmr_solve_many(h, [As[k]], [Fs[k]], [bs[k]], [x1], 1e-8, 1000)
        assert torch.equal(x1, xs[k]) and i1[0] == its[k] and r1[0] == res[k]
        rp, ci, v, bl = pats[k]
        S = oracle.Sym(rp, ci, bl, 0, 1.0)
        xo, _, ito = oracle.sqmr(rp, ci, v, bs[k].cpu().numpy(), S.factor(v), 1e-8, 1000)
        assert abs(int(its[k]) - ito) <= max(4, 0.05 * ito)
