"""KKT assembly of an interior-point iteration (culipx_kkt_assembly_*):
K = [[diag(d) + delta I, A'], [A, -gamma I]], d = s / x or given, as full
symmetric CSR.  Structure and values must equal the numpy restatement
(oracle.kkt_assemble) bit for bit, and rebuilding the seeded KKT generator's K
from its own A block and diagonal must give that K exactly."""
import numpy as np
import pytest

import culip_b200 as cb
import oracle


def _split_kkt(rp, ci, v, n, m):
    """A (m x n CSR), diag(H + delta) and the dual diagonal of a generated K."""
    rows = np.repeat(np.arange(n + m), np.diff(rp))
    sel = (rows >= n) & (ci < n)
    a_rows = rows[sel] - n
    a_rp = np.zeros(m + 1, np.int64)
    np.add.at(a_rp, a_rows + 1, 1)
    a_rp = np.cumsum(a_rp).astype(np.int32)
    diag = v[rows == ci]
    return a_rp, ci[sel].astype(np.int32), v[sel], diag[:n], -diag[n:]


def _random_a(m, n, seed, density=0.02):
    """Ragged A: some empty rows and columns, sorted unique columns per row."""
    rng = np.random.default_rng(seed)
    rp, ci = [0], []
    for i in range(m):
        k = 0 if i % 7 == 3 else int(rng.integers(0, max(2, int(density * n) * 2)))
        cols = np.unique(rng.integers(0, max(n - 3, 1), k))  # the last columns stay empty
        ci.extend(cols.tolist())
        rp.append(len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), rng.standard_normal(len(ci))


def test_oracle_rebuilds_generated_kkt():
    cfg = cb.KKT_CONFIGS["small"]
    n, m = cfg["n"], cfg["m"]
    rp, ci, v = cb.kkt_generate(n, m, cfg["nnz_per_col"], cfg["band_half"], cfg["hmin"], cfg["hmax"])
    a_rp, a_ci, a_v, hd, gd = _split_kkt(rp, ci, v, n, m)
    assert np.all(gd == gd[0])
    krp, kci, kv = oracle.kkt_assemble(m, n, a_rp, a_ci, a_v, d=hd, delta=0.0, gamma=float(gd[0]))
    assert np.array_equal(krp, rp) and np.array_equal(kci, ci) and np.array_equal(kv, v)


def test_oracle_structure_rules():
    a_rp, a_ci, a_v = _random_a(40, 60, 1)
    x = np.linspace(1.0, 2.0, 60)
    s = np.linspace(3.0, 0.5, 60)
    krp, kci, kv = oracle.kkt_assemble(40, 60, a_rp, a_ci, a_v, x=x, s=s, delta=1e-8, gamma=1e-6)
    N = 100
    assert krp[-1] == 2 * len(a_ci) + N
    for r in range(N):
        c = kci[krp[r]:krp[r + 1]]
        assert np.all(np.diff(c) > 0) and r in c
    K = np.zeros((N, N))
    for r in range(N):
        K[r, kci[krp[r]:krp[r + 1]]] = kv[krp[r]:krp[r + 1]]
    assert np.array_equal(K, K.T)
    assert np.array_equal(np.diag(K)[:60], s / x + 1e-8) and np.all(np.diag(K)[60:] == -1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["xs", "d"])
@pytest.mark.parametrize("precision", [cb.F64, cb.F32])
def test_gpu_assembly_matches_oracle(mode, precision):
    torch = pytest.importorskip("torch")
    m, n = 300, 500
    a_rp, a_ci, a_v = _random_a(m, n, 7)
    rng = np.random.default_rng(3)
    x = 10.0 ** rng.uniform(-4, 4, n)
    s = 10.0 ** rng.uniform(-4, 4, n)
    d = 10.0 ** rng.uniform(-6, 6, n)
    h = cb.Handle(0)
    K = cb.KktAssembly(h, m, n, torch.from_numpy(a_rp).cuda(), torch.from_numpy(a_ci).cuda())
    kw = dict(x=x, s=s) if mode == "xs" else dict(d=d)
    krp, kci, kv = oracle.kkt_assemble(m, n, a_rp, a_ci, a_v, delta=1e-8, gamma=2e-8, **kw)
    grp, gci = K.structure()
    assert np.array_equal(grp, krp) and np.array_equal(gci, kci)
    dt = torch.float64 if precision == cb.F64 else torch.float32
    out = torch.zeros(K.nnz, dtype=dt, device="cuda")
    dkw = {k: torch.from_numpy(val).cuda() for k, val in kw.items()}
    K.assemble(torch.from_numpy(a_v).cuda(), out, delta=1e-8, gamma=2e-8, **dkw)
    got = out.cpu().numpy()
    want = kv if precision == cb.F64 else kv.astype(np.float32)
    assert np.array_equal(got, want)


@pytest.mark.gpu
def test_gpu_assembly_rebuilds_generated_kkt_and_solves():
    """The small workload's K rebuilt on the device from its A block and
    diagonal, analysed from the exported structure, factored and solved."""
    torch = pytest.importorskip("torch")
    cfg = cb.KKT_CONFIGS["small"]
    n, m = cfg["n"], cfg["m"]
    rp, ci, v = cb.kkt_generate(n, m, cfg["nnz_per_col"], cfg["band_half"], cfg["hmin"], cfg["hmax"])
    a_rp, a_ci, a_v, hd, gd = _split_kkt(rp, ci, v, n, m)
    h = cb.Handle(0)
    K = cb.KktAssembly(h, m, n, torch.from_numpy(a_rp).cuda(), torch.from_numpy(a_ci).cuda())
    krp, kci = K.structure()
    assert np.array_equal(krp, rp) and np.array_equal(kci, ci)
    kv = torch.zeros(K.nnz, dtype=torch.float64, device="cuda")
    K.assemble(torch.from_numpy(a_v).cuda(), kv, d=torch.from_numpy(hd).cuda(), delta=0.0, gamma=float(gd[0]))
    assert np.array_equal(kv.cpu().numpy(), v)
    bs = cb.kkt_blocking(n, m, cfg["block"])
    P = cb.Pattern(h, krp, kci, bs, 0, 1.0, cb.F64)
    F = cb.Factor(P)
    F.compute(kv)
    A = cb.CsrOperator(h, torch.from_numpy(krp).cuda(), torch.from_numpy(kci).cuda(), kv)
    b = cb.normal_vector(cb.SEED + 1, n + m)
    xg = torch.zeros(n + m, dtype=torch.float64, device="cuda")
    res, its, st = cb.sqmr_solve(h, A, F, torch.from_numpy(b).cuda(), xg, 1e-8, 1000)
    import scipy.sparse as sp

    Ks = sp.csr_matrix((v, ci, rp), shape=(n + m, n + m))
    assert np.linalg.norm(b - Ks @ xg.cpu().numpy()) <= 1e-5 * np.linalg.norm(b)


@pytest.mark.gpu
def test_gpu_assembly_rejects_bad_structure():
    torch = pytest.importorskip("torch")
    h = cb.Handle(0)
    rp = torch.tensor([0, 2, 3], dtype=torch.int32, device="cuda")
    bad_sorted = torch.tensor([3, 1, 0], dtype=torch.int32, device="cuda")
    with pytest.raises(cb.CulipxError):
        cb.KktAssembly(h, 2, 5, rp, bad_sorted)
    bad_range = torch.tensor([0, 7, 1], dtype=torch.int32, device="cuda")
    with pytest.raises(cb.CulipxError):
        cb.KktAssembly(h, 2, 5, rp, bad_range)
    # empty A: K = diag
    e = torch.zeros(1, dtype=torch.int32, device="cuda")
    K = cb.KktAssembly(h, 0, 4, e, e[:0])
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    K.assemble(None, out, d=torch.arange(4, dtype=torch.float64, device="cuda"), delta=1.0)
    assert out.cpu().tolist() == [1.0, 2.0, 3.0, 4.0]
