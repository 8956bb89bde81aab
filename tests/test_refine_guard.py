"""FP64 refinement returns its best iterate and stops when corrections stop
helping.

With tol = 0 the refinement can never pass its test, so every loop runs
until two corrections in a row fail to lower the smallest ||b - K x|| (the
residual reached the rounding floor) and must then stop with CULIPX_STALLED,
returning the iterate of smallest residual.  The refinement is deterministic
(fixed-order reductions), so that x must be bit for bit the x of a run
capped at the correction that produced it, which ends with CULIPX_MAXIT.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import culip_b200 as cb
from culip_b200 import _capi as capi
from problems import kkt

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MAX_REFINE = 40
PATIENCE = 2  # non-improving corrections in a row that end the loop


@pytest.fixture(scope="module")
def small():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    h = cb.Handle(0)
    rp, ci, v, bs = kkt("small")
    n = len(rp) - 1
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F32)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v.astype(np.float32)).cuda())
    A = cb.CsrOperator(h, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    K = sp.csr_matrix((v, ci, rp))
    return dict(h=h, rp=rp, ci=ci, v=v, bs=bs, n=n, P=P, F=F, A=A, K=K)


def _refine(s, b, max_refine):
    x = torch.zeros(s["n"], dtype=torch.float64, device="cuda")
    rel, its, steps, st = cb.sqmr_refine(s["h"], s["A"], s["F"], torch.from_numpy(b).cuda(), x, 0.0, 1e-6, 1000,
                                         max_refine)
    return rel, its, steps, st, x.cpu().numpy()


def test_refine_stalls_with_best_iterate(small):
    b = cb.normal_vector(cb.SEED + 1, small["n"])
    rel, its, steps, st, x = _refine(small, b, MAX_REFINE)
    assert st == capi.STALLED and PATIENCE + 1 <= steps < MAX_REFINE
    # capped at the correction that gave the best iterate
    rel1, its1, steps1, st1, x1 = _refine(small, b, steps - PATIENCE)
    assert st1 == capi.MAXIT and steps1 == steps - PATIENCE
    assert np.array_equal(x, x1) and rel == rel1
    true_rel = np.linalg.norm(b - small["K"] @ x) / np.linalg.norm(b)
    assert rel < 1e-12 and true_rel < 1e-12


@pytest.mark.parametrize("nrhs", [1, 3])
def test_refine_multi_stalls_per_column(small, nrhs):
    rng = np.random.default_rng(40 + nrhs)
    B = rng.standard_normal((nrhs, small["n"])) * (10.0 ** np.arange(nrhs))[:, None]

    def run(max_refine):
        X = torch.zeros((nrhs, small["n"]), dtype=torch.float64, device="cuda")
        out = cb.sqmr_refine_multi(small["h"], small["A"], small["F"], torch.from_numpy(B).cuda(), X, 0.0, 1e-6, 1000,
                                   max_refine)
        return out + (X.cpu().numpy(),)

    rel, its, steps, st, X = run(MAX_REFINE)
    assert (st == capi.STALLED).all() and (steps > PATIENCE).all() and (steps < MAX_REFINE).all()
    cap = int(steps.max()) - PATIENCE
    rel1, its1, steps1, st1, X1 = run(cap)
    for r in range(nrhs):
        assert np.array_equal(X[r], X1[r]) and rel[r] == rel1[r]
        assert st1[r] == (capi.STALLED if steps[r] <= cap else capi.MAXIT)
        true_rel = np.linalg.norm(B[r] - small["K"] @ X[r]) / np.linalg.norm(B[r])
        assert true_rel < 1e-12


def test_batch_refine_stalls_per_system():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from test_batch import _rhs, _systems

    h = cb.Handle(0)
    syst = _systems(4, seed=23)
    rp, ci, v, bs, off = cb.union_systems(syst)
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F32, system_row_offsets=off)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v.astype(np.float32)).cuda())
    A = cb.CsrOperator(h, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    b = np.concatenate(_rhs(syst, range(4)))
    B = cb.Batch(P, off)

    def run(max_refine):
        x = torch.zeros(len(rp) - 1, dtype=torch.float64, device="cuda")
        out = cb.batch_sqmr_refine(B, A, F, torch.from_numpy(b).cuda(), x, 0.0, 1e-6, 1000, max_refine)
        return out + (x.cpu().numpy(),)

    rel, its, steps, st, x = run(MAX_REFINE)
    assert (st == capi.STALLED).all() and (steps < MAX_REFINE).all()
    # capped at the last system's best correction: the systems that stalled
    # earlier are identical, the last one ends with MAXIT on the same x
    cap = int(steps.max()) - PATIENCE
    rel1, its1, steps1, st1, x1 = run(cap)
    for k, (srp, sci, sv, sbs) in enumerate(syst):
        seg = slice(off[k], off[k + 1])
        if steps[k] <= cap:
            assert st1[k] == capi.STALLED and np.array_equal(x[seg], x1[seg])
        else:
            assert st1[k] == capi.MAXIT and np.array_equal(x[seg], x1[seg]) and rel[k] == rel1[k]
        K = sp.csr_matrix((sv, sci, srp))
        assert np.linalg.norm(b[seg] - K @ x[seg]) / np.linalg.norm(b[seg]) < 1e-12


def test_server_refine_stalls():
    """Server requests with tol 0: every right-hand side ends STALLED at the
    rounding floor, never with a residual above the plain solve's."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rp, ci, v = cb.kkt_generate(400, 200, 6, 16, 1e-3, 1e3, seed=cb.SEED + 5410)
    bs = cb.kkt_blocking(400, 200, 16)
    rng = np.random.default_rng(9)
    b = rng.standard_normal((len(rp) - 1, 2))
    s = cb.Server(0, 0, 1, 2, 0.0, 200)
    s.set_refine(MAX_REFINE, 1e-6)
    pid = s.add_pattern(rp, ci, bs, cb.F32)
    rid = s.submit(pid, v, b)
    while s.progress(wait=True) == 0:
        pass
    x, its, status, lat = s.result(rid)
    K = sp.csr_matrix((v, ci, rp))
    for r in range(2):
        assert status[r] == capi.STALLED
        assert np.linalg.norm(b[:, r] - K @ x[:, r]) / np.linalg.norm(b[:, r]) < 1e-12
