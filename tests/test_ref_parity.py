"""GPU parity against the reference itself: culip's own BlockiLDLt, SQMR and
CSR operator, compiled from its sources for sm_100a (oracle/build_ref.py ->
oracle/_ref/ref_dump), run on the same inputs as the culipx path.

* The factor -- every block's values and sparsity, D, the pivot flags and the
  pivoting permutation -- must equal the reference's bit for bit, on the
  benchmarked scale workload (n = 200000, m = 100000, 32-row blocks, BK)
  included, and on scrambled systems (2x2 pivots, swaps, deep level
  schedules).  With fill levels 1-2 the reference's leftover grants race
  (replayed into the oracle) and its own runs also differ in the last bits
  of a few blocks: there the sparsity, pivots and permutation are exact and
  the values within 1e-9 of each block's largest entry (D^-1 b within 1e-7).
* D^-1 b is a per-row formula: bit for bit.  The triangular sweeps: the
  reference sums each row's terms with atomicAdd (block_ildlt_kernels.impl.cuh
  k_solve_blocks_*), so its own results vary in the last bits; within 1e-14
  on natural-order systems, and a backward error within 1e-13 against the
  (bit-identical) factor on scrambled ones.
* SQMR: the iteration counts agree within 4 (8 on the 1000-iteration scale
  solve, where neither converges) and the true relative residuals within 5 %
  (converged small system: rounding-level residuals) / 1 % (scale).
* The reference's apps/block_ildlt driver, unmodified, compiled against the
  culip_la.hpp facade (oracle/_ref/culip-block-ildlt-b200) prints what the
  same driver built on the reference prints: iterations within 4, the
  converged residuals and error within a factor 2.
"""
import os
import re
import subprocess

import numpy as np
import pytest

import culip_b200 as cb
import oracle
from oracle import ref
from problems import kkt, scrambled_kkt

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def handle():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not ref.available():
        pytest.skip("reference build (oracle/_ref) not present")
    return cb.Handle(0)


def _gpu_factor(handle, rp, ci, v, bs, pivot, precision, fill_level=0, is_piv=None):
    dt = np.float64 if precision == cb.F64 else np.float32
    P = cb.Pattern(handle, rp, ci, bs, fill_level, 1.0, precision)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v.astype(dt)).cuda(), is_piv=is_piv, pivot=pivot)
    pe = P.export()
    rows = np.repeat(np.arange(len(pe["coarse_off"]) - 1), np.diff(pe["coarse_off"]))
    return P, F, ref.canonical_export(F.export(), rows, pe["coarse_col"], pe["fmt"])


def _assert_blocks_equal(mine, theirs, rtol=0.0):
    """Same blocks, formats and sparsity; values bit for bit (rtol 0) or
    within rtol of each block's largest entry."""
    assert set(mine) == set(theirs)
    for key, (fr, nr, _gr, ir, vr) in theirs.items():
        fm, nm, _gm, im, vm = mine[key]
        assert fm == fr, key
        assert np.array_equal(im, ir), key
        if rtol == 0.0:
            assert np.array_equal(vm, vr), key
        else:
            scale = float(np.max(np.abs(vr))) if len(vr) else 0.0
            assert np.max(np.abs(vm - vr), initial=0.0) <= rtol * scale, key


CASES = {
    "small_f64_bk": (lambda: kkt("small"), cb.PIV_BK, cb.F64, 0),
    "small_f32_bk": (lambda: kkt("small"), cb.PIV_BK, cb.F32, 0),
    "small_f64_static": (lambda: kkt("small"), cb.PIV_STATIC, cb.F64, 0),
    "banded_b32_f64_bk": (lambda: kkt("small", block=32, band_half=16), cb.PIV_BK, cb.F64, 0),
    "scrambled_f64_bk": (lambda: scrambled_kkt(), cb.PIV_BK, cb.F64, 0),
    "scrambled_f32_bk": (lambda: scrambled_kkt(seed=11), cb.PIV_BK, cb.F32, 0),
    "scrambled9_f64_bk": (lambda: scrambled_kkt(seed=9), cb.PIV_BK, cb.F64, 0),
    "scrambled_f64_static": (lambda: scrambled_kkt(seed=5), cb.PIV_STATIC, cb.F64, 0),
    "scrambled_f64_bk_fill1": (lambda: scrambled_kkt(seed=3), cb.PIV_BK, cb.F64, 1),
    "scrambled_f64_bk_fill2": (lambda: scrambled_kkt(seed=4), cb.PIV_BK, cb.F64, 2),
    "scale_f64_bk": (lambda: kkt("scale"), cb.PIV_BK, cb.F64, 0),
}


def _u_matrix(E, S, bs, n):
    """U of an exported factor as a sparse matrix: the off-diagonal blocks and
    the upper triangles of the pivot tiles (what the sweeps read)."""
    import scipy.sparse as sp

    bs = np.asarray(bs)
    if bs[-1] != n:
        bs = np.concatenate([bs, [n]])
    rows, cols, vals = [], [], []
    for q in range(S.coarse_nnz):
        I, J = int(S.blk_row[q]), int(S.blk_col[q])
        w = bs[J + 1] - bs[J]
        e0, e1 = E["blk_off"][q], E["blk_off"][q + 1]
        idx, v = E["idx"][e0:e1], E["val"][e0:e1].astype(np.float64)
        r, c = bs[I] + idx // w, bs[J] + idx % w
        keep = (v != 0) & ((c >= r) if I == J else True)
        rows.append(r[keep]), cols.append(c[keep]), vals.append(v[keep])
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))


def _backward_error(U, perm, b, y, stage):
    """max |c - T y| / max (|T| |y|) of the triangular solve behind a left
    (T = U', c = b[perm]) or right (T = U, c = b, y read as x[perm]) apply."""
    y = y.astype(np.float64)
    if stage == cb.LEFT:
        T, c, t = U.T, b[perm], y
    else:
        T, c, t = U, b, y[perm]
    r = c - T @ t
    return np.max(np.abs(r)) / np.max(abs(T) @ np.abs(t))


def _assert_applies(apply, R, b, dt, direct, U=None, perm=None, mtol=0.0):
    """D^-1 b bit for bit; the sweeps within 1e-14 (FP32: 1e-6) of the
    reference's on natural-order systems.  On scrambled systems (entries up to
    1e8, long cancelling sums) the reference's atomicAdd order moves its result
    further; there both results must solve the same triangular system to
    rounding accuracy (backward error 1e-13, FP32 1e-5)."""
    tol = 1e-14 if dt == np.float64 else 1e-6
    btol = 1e-13 if dt == np.float64 else 1e-5
    for stage, key in ((cb.LEFT, "apply_left"), (cb.MIDDLE, "apply_middle"), (cb.RIGHT, "apply_right")):
        y = apply(stage)
        yr = R[key]
        if stage == cb.MIDDLE:
            if mtol:
                assert np.linalg.norm(y.astype(float) - yr) <= mtol * np.linalg.norm(yr), key
            else:
                assert np.array_equal(y, yr), key
        elif direct:
            assert np.linalg.norm(y.astype(float) - yr) <= tol * np.linalg.norm(yr), key
        else:
            bb = b.astype(dt).astype(np.float64)
            assert _backward_error(U, perm, bb, y, stage) <= btol, key
            assert _backward_error(U, perm, bb, yr, stage) <= btol, key


@pytest.mark.parametrize("case", list(CASES))
def test_factor_and_applies_match_reference(handle, case):
    """Bit for bit.  Where blocks outgrow their capacity, the reference's CTAs
    race for the leftover slots (k_apply_block_dual_dropping,
    block_ildlt_kernels.impl.cuh:1949-2008) and which request of a level wins
    depends on the hardware; the oracle replays the reference's grants then,
    and the GPU path equals the oracle (its own, deterministic grants)."""
    make, pivot, precision, fill = CASES[case]
    rp, ci, v, bs = make()
    n = len(rp) - 1
    dt = np.float64 if precision == cb.F64 else np.float32
    # with fill, the reference varies between its own runs: up to 30 of its
    # grants, and (grants replayed) the last bits of a few blocks
    rtol = 0.0 if fill == 0 else 1e-9
    b = cb.normal_vector(cb.SEED + 1, n)
    R = ref.run(rp, ci, v, bs, b, precision=1 if precision == cb.F64 else 0, pivot=pivot, fill_level=fill,
                max_it=0)
    theirs = ref.canonical_blocks(R)
    P, F, mine = _gpu_factor(handle, rp, ci, v, bs, pivot, precision, fill)
    S = oracle.Sym(rp, ci, bs, fill, 1.0, dtype=dt)
    ref_grants = np.array([theirs[(int(S.blk_row[q]), int(S.blk_col[q]))][2] for q in range(S.coarse_nnz)],
                          np.int32)
    # the reference's own numerics, its grant decisions given
    OFr = S.factor(v.astype(dt), pivot=pivot, forced_grants=ref_grants)
    Er = OFr.export()
    _assert_blocks_equal(ref.canonical_export(Er, S.blk_row, S.blk_col, S.fmt), theirs, rtol)
    for k in ("is_piv", "perm"):
        assert np.array_equal(Er[k], R[k]), k
    assert np.allclose(Er["tri"], R["tri"], rtol=rtol, atol=0.0) if rtol else np.array_equal(Er["tri"], R["tri"])
    direct = not case.startswith("scrambled")
    U = None if direct else _u_matrix(Er, S, bs, n)
    _assert_applies(lambda st: OFr.apply(st, b.astype(dt)), R, b, dt, direct, U, Er["perm"], 1e2 * rtol)
    # the GPU path against the oracle with its own grants, bit for bit
    E = F.export()
    Eo = S.factor(v.astype(dt), pivot=pivot).export()
    for k in ("blk_off", "idx", "val", "tri", "is_piv", "perm", "got_extra"):
        assert np.array_equal(E[k], Eo[k]), k
    bt = torch.from_numpy(b.astype(dt)).cuda()
    if np.array_equal(E["got_extra"], ref_grants):
        # the same decisions: the GPU factor and applies against the reference directly
        _assert_blocks_equal(mine, theirs, rtol)
        for k in ("is_piv", "perm"):
            assert np.array_equal(E[k], R[k]), k
        assert np.allclose(E["tri"], R["tri"], rtol=rtol, atol=0.0) if rtol else np.array_equal(E["tri"], R["tri"])
        _assert_applies(lambda st: F.apply(st, bt).cpu().numpy(), R, b, dt, direct, U, Er["perm"], 1e2 * rtol)


@pytest.mark.parametrize("name,its_tol,rtol,restol", [("small", 4, 5e-2, 0.2), ("scale", 8, 1e-2, 5e-2)])
def test_sqmr_matches_reference(handle, name, its_tol, rtol, restol):
    """small converges (true relres ~5e-6 and the last quasi-residual ~1e-7,
    both set by rounding at the stopping iteration: 5 % / 20 %); scale runs
    into max_it on both sides (1 % / 5 %)"""
    rp, ci, v, bs = kkt(name)
    n = len(rp) - 1
    b = cb.normal_vector(cb.SEED + 1, n)
    R = ref.run(rp, ci, v, bs, b, precision=1, pivot=cb.PIV_BK, tol=1e-8, max_it=1000)
    P = cb.Pattern(handle, rp, ci, bs, 0, 1.0, cb.F64)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v).cuda())
    A = cb.CsrOperator(handle, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    res, its, _ = cb.sqmr_solve(handle, A, F, torch.from_numpy(b).cuda(), x, 1e-8, 1000)
    import scipy.sparse as sp

    K = sp.csr_matrix((v, ci, rp), shape=(n, n))
    relres = np.linalg.norm(b - K @ x.cpu().numpy()) / np.linalg.norm(b)
    assert abs(its - R["iterations"]) <= its_tol
    assert abs(relres - R["true_relres"]) <= rtol * R["true_relres"]
    assert abs(res - R["residual"]) <= restol * R["residual"]


def _write_mtx_system(d, rp, ci, v, bs):
    n = len(rp) - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    with open(os.path.join(d, "K.mtx"), "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate real general\n{n} {n} {len(ci)}\n")
        f.writelines(f"{i + 1} {j + 1} {float(x)!r}\n" for i, j, x in zip(rows.tolist(), ci.tolist(), v.tolist()))

    def vec(name, a):
        with open(os.path.join(d, name), "w") as f:
            f.write(f"%%MatrixMarket matrix array integer general\n{len(a)} 1\n")
            f.writelines(f"{int(x)}\n" for x in a)

    vec("perm.mtx", np.arange(n))
    vec("blocks.mtx", np.concatenate([bs[:-1] if bs[-1] == n else bs, [n]]))
    vec("piv.mtx", np.ones(n, np.int64))


def _driver_numbers(out):
    m = re.search(r"SQMR: residual (\S+) after (\d+) iterations", out)
    e = re.search(r"True relative error: (\S+)", out)
    r = re.search(r"True relative residual: (\S+)", out)
    assert m and e and r, out[-2000:]
    return float(m.group(1)), int(m.group(2)), float(e.group(1)), float(r.group(1))


def test_unmodified_driver_on_the_facade(handle, tmp_path):
    """apps/block_ildlt as the reference ships it, built against culip_la.hpp,
    gives what the same driver built on the reference gives: the iteration
    count within 4, residuals and error within a factor 2."""
    mine_exe = ref.REF_DRIVER + "-b200"
    if not (os.path.exists(mine_exe) and os.path.exists(ref.REF_DRIVER)):
        pytest.skip("drivers not built")
    rp, ci, v, bs = kkt("small")
    _write_mtx_system(str(tmp_path), rp, ci, v, bs)
    args = [str(tmp_path / "K.mtx"), str(tmp_path / "perm.mtx"), str(tmp_path / "blocks.mtx"),
            str(tmp_path / "piv.mtx"), "1", "1", "0", "1.0", "0.0"]
    outs = []
    for exe in (ref.REF_DRIVER, mine_exe):
        r = subprocess.run([exe, *args], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (exe, r.stdout[-2000:], r.stderr[-2000:])
        outs.append(_driver_numbers(r.stdout))
    (rres, rits, rerr, rrel), (mres, mits, merr, mrel) = outs
    # the reference's triangular sweeps sum with atomicAdd, so its own
    # iteration count moves by a few between runs (224 and 228 seen)
    assert abs(mits - rits) <= 4
    # both runs converge; at the (lagged, every 4th iteration) stop the residual
    # and the error are rounding-level and move with the stopping iteration
    # (2.6e-7 vs 3.4e-7 seen for the error): within a factor 2
    for mine, theirs in ((mrel, rrel), (merr, rerr), (mres, rres)):
        assert theirs / 2 <= mine <= 2 * theirs + 1e-12
