"""GPU parity at the benchmarked sizes, against the CPU oracle.

The scale workload (n = 200000, m = 100000: N = 300000, 6 entries per column
of A, H log-uniform in [1e-6, 1e6], 32-row blocks, BK, level-0 fill) is the
one bench.py times; here it is factored and solved on the GPU and by the
oracle on the same seeded input:

* factor (values, D, pivot flags, permutation, granted slots): bit for bit;
* the three preconditioner stages: bit for bit (both sum each row's terms in
  increasing column order);
* SQMR capped at 20 and 100 iterations: the same iteration count, x within
  1e-12 / 1e-10.  The GPU's recurrence is re-associated (1/delta after the
  linear sweep, the p / x update one phase later, fixed-tree reductions), so
  its roundings differ from the oracle's serial sums and the gap grows with
  the iterations;
* 1000 iterations (the benchmark's solve; neither converges on this late-IPM
  system): the true relative residuals agree within 5e-3 (1.4465 vs 1.4482 on
  the B200; the reference's own GPU code gives 1.4469).

The mixed-precision construction (n = 1e6, m = 5e5) is checked on a tenth of
its size with an FP32 factor, bit for bit; the GPU SpMV on the reference's
spmv_A / spmv_K fixtures with the assertions of tests/la/test_spmv.cc:150-168
(their rows average more than 16 entries, so the product runs warp per row
and is not bit for bit with the oracle's serial row sums).
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import culip_b200 as cb
from culip_b200 import _capi as capi
import oracle
from problems import kkt

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def scale():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    h = cb.Handle(0)
    rp, ci, v, bs = kkt("scale")
    n = len(rp) - 1
    b = cb.normal_vector(cb.SEED + 1, n)
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F64)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v).cuda())
    S = oracle.Sym(rp, ci, bs, 0, 1.0)
    OF = S.factor(v)
    A = cb.CsrOperator(h, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    return dict(h=h, rp=rp, ci=ci, v=v, bs=bs, b=b, n=n, P=P, F=F, S=S, OF=OF, A=A)


def test_scale_factor_exact(scale):
    oe, ge = scale["OF"].export(), scale["F"].export()
    for k in ("blk_off", "blk_nnz", "idx", "is_piv", "perm", "got_extra"):
        assert np.array_equal(oe[k], ge[k]), k
    assert np.array_equal(oe["val"], ge["val"])
    assert np.array_equal(oe["tri"], ge["tri"])


@pytest.mark.parametrize("stage", [cb.LEFT, cb.MIDDLE, cb.RIGHT])
def test_scale_applies_exact(scale, stage):
    b = scale["b"]
    y = scale["F"].apply(stage, torch.from_numpy(b).cuda()).cpu().numpy()
    assert np.array_equal(y, scale["OF"].apply(stage, b))


@pytest.mark.parametrize("cap,xtol", [(20, 1e-12), (100, 1e-10)])
def test_scale_sqmr_capped(scale, cap, xtol):
    s = scale
    x = torch.zeros(s["n"], dtype=torch.float64, device="cuda")
    res, its, st = cb.sqmr_solve(s["h"], s["A"], s["F"], torch.from_numpy(s["b"]).cuda(), x, 1e-8, cap)
    xo, reso, ito = oracle.sqmr(s["rp"], s["ci"], s["v"], s["b"], s["OF"], 1e-8, cap)
    assert its == ito == cap
    xg = x.cpu().numpy()
    assert np.linalg.norm(xg - xo) <= xtol * np.linalg.norm(xo)
    assert abs(res - reso) <= 1e-8 * reso


def test_scale_sqmr_1000_true_relres(scale):
    s = scale
    K = sp.csr_matrix((s["v"], s["ci"], s["rp"]), shape=(s["n"], s["n"]))
    x = torch.zeros(s["n"], dtype=torch.float64, device="cuda")
    _, its, _ = cb.sqmr_solve(s["h"], s["A"], s["F"], torch.from_numpy(s["b"]).cuda(), x, 1e-8, 1000)
    xo, _, ito = oracle.sqmr(s["rp"], s["ci"], s["v"], s["b"], s["OF"], 1e-8, 1000)
    with open(os.path.join(GOLDEN, "sqmr_iterations_scale.txt")) as f:
        assert ito == int(f.read().split()[0])
    assert its == ito
    nb = np.linalg.norm(s["b"])
    rg = np.linalg.norm(s["b"] - K @ x.cpu().numpy()) / nb
    ro = np.linalg.norm(s["b"] - K @ xo) / nb
    assert abs(rg - ro) <= 5e-3 * ro


def test_scale_refine_never_worse_than_start(scale):
    """Refinement on the scale workload: its 1000-iteration correction leaves
    a true relative residual near 1.45, above the 1.0 of x = 0.  The
    refinement returns its best iterate, so its relres is at most 1.0 and is
    the true residual of the returned x, and it stops (STALLED) once
    corrections stop helping instead of running to max_refine."""
    s = scale
    x = torch.full((s["n"],), 7.0, dtype=torch.float64, device="cuda")
    rel, its, steps, st = cb.sqmr_refine(s["h"], s["A"], s["F"], torch.from_numpy(s["b"]).cuda(), x, 1e-8, 1e-8, 1000,
                                         6)
    assert st in (capi.STALLED, capi.MAXIT) and steps >= 2 and its <= 1000 * steps
    assert rel <= 1.0
    K = sp.csr_matrix((s["v"], s["ci"], s["rp"]), shape=(s["n"], s["n"]))
    xh = x.cpu().numpy()
    true_rel = np.linalg.norm(s["b"] - K @ xh) / np.linalg.norm(s["b"])
    assert abs(true_rel - rel) <= 1e-9 * rel
    if rel == 1.0:
        assert not xh.any()


def test_mixed_construction_tenth_fp32_factor_exact():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    h = cb.Handle(0)
    rp, ci, v, bs = kkt("mixed", n=100000, m=50000)
    S = oracle.Sym(rp, ci, bs, 0, 1.0, dtype=np.float32)
    oe = S.factor(v.astype(np.float32)).export()
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F32)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v.astype(np.float32)).cuda())
    ge = F.export()
    for k in ("blk_off", "idx", "is_piv", "perm", "got_extra"):
        assert np.array_equal(oe[k], ge[k]), k
    assert np.array_equal(oe["val"], ge["val"])
    assert np.array_equal(oe["tri"], ge["tri"])


@pytest.mark.parametrize("name", ["A", "K"])
@pytest.mark.parametrize("transpose", [False, True])
def test_gpu_spmv_on_reference_fixtures(name, transpose):
    """tests/la/test_spmv.cc:150-168: y = A x (and A' x) with x = 0.1, FP64,
    against the exact product to 1e-10."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    d = np.load(os.path.join(GOLDEN, f"spmv_{name}.npz"))
    m, n = int(d["m"]), int(d["n"])
    h = cb.Handle(0)
    A = cb.CsrOperator(h, torch.from_numpy(d["rowptr"]).cuda(), torch.from_numpy(d["colidx"]).cuda(),
                       torch.from_numpy(d["val"]).cuda(), ncols=n, explicit_transpose=transpose)
    M = sp.csr_matrix((d["val"], d["colidx"], d["rowptr"]), shape=(m, n))
    x = np.full(m if transpose else n, 0.1)
    y = torch.zeros(n if transpose else m, dtype=torch.float64, device="cuda")
    y = A.spmv(torch.from_numpy(x).cuda(), y, transpose=transpose).cpu().numpy()
    exact = (M.T @ x) if transpose else (M @ x)
    assert np.allclose(y, exact, rtol=1e-10, atol=1e-10)
