"""FP32 factors invert ill-conditioned 2x2 pivots in FP64.

A 2x2 pivot whose ratio |d11 d22 - d12^2| / (|d11 d22| + d12^2) is below the
bound (default 1e-3) is solved in double in the pivot-tile step
(d_ldlt_2x2_step, block_ildlt_kernels.impl.cuh:589-675), the off-diagonal
solve (d_left_solve_with_D_Ut, :1489-1570) and the D apply (k_solve_D,
helper_kernels.impl.cuh:720-774), each result rounded to float once.  The
planted problem (tests/problems.py:planted_pairs) has statically pivoted
pairs with ratio about 5e-6 at level 0:

* oracle, on the CPU: the FP32 factor with the FP64 inversion is within 1e-6
  of the FP64 factor; in float throughout (bound 0, the reference's
  arithmetic) it is off by more than 1 %;
* GPU against the oracle, bit for bit, for both bounds (factor and applies);
* GPU with bound 0 against the reference's own float build, bit for bit.
"""
import numpy as np
import pytest

import culip_b200 as cb
import oracle
from problems import planted_pairs


def _factor_err(E32, E64):
    """||U32 - U64|| / ||U64|| over every block's stored entries (an entry
    one factor dropped as zero counts as 0 there)."""
    d = 0.0
    for q in range(len(E64["blk_off"]) - 1):
        a0, a1 = E32["blk_off"][q], E32["blk_off"][q + 1]
        b0, b1 = E64["blk_off"][q], E64["blk_off"][q + 1]
        u = dict(zip(E64["idx"][b0:b1].tolist(), E64["val"][b0:b1].tolist()))
        for i, x in zip(E32["idx"][a0:a1].tolist(), E32["val"][a0:a1].astype(np.float64).tolist()):
            u[i] = u.get(i, 0.0) - x
        d += sum(t * t for t in u.values())
    return np.sqrt(d) / np.linalg.norm(E64["val"])


def test_oracle_fp64_inversion_recovers_fp32_factor():
    rp, ci, v, bs, ip = planted_pairs()
    E64 = oracle.Sym(rp, ci, bs, 0, 1.0).factor(v, is_piv=ip, pivot=cb.PIV_STATIC).export()
    S32 = oracle.Sym(rp, ci, bs, 0, 1.0, dtype=np.float32)
    wide = S32.factor(v.astype(np.float32), is_piv=ip, pivot=cb.PIV_STATIC).export()
    plain = S32.factor(v.astype(np.float32), is_piv=ip, pivot=cb.PIV_STATIC, pivot_fp64=0.0).export()
    for k in ("blk_off", "is_piv", "perm"):
        assert np.array_equal(wide[k], E64[k]) and np.array_equal(plain[k], E64[k]), k
    assert np.array_equal(wide["idx"], E64["idx"])
    assert _factor_err(wide, E64) < 1e-6
    assert _factor_err(plain, E64) > 1e-2
    # the pairs really are below the bound, and their D is stored unchanged
    # (the level-1 rows' D are Schur complements of the two factors' U)
    t = E64["tri"].reshape(-1, 3)
    half = (len(rp) - 1) // 2
    d11, d12, d22 = t[0:half:2, 1], t[0:half:2, 2], t[1:half:2, 1]
    ratio = np.abs(d11 * d22 - d12 * d12) / (np.abs(d11 * d22) + d12 * d12)
    assert (ratio < 1e-4).all()
    assert np.array_equal(wide["tri"][:3 * half], plain["tri"][:3 * half])


def test_oracle_fp64_bound_leaves_fp64_and_bk_factors_alone():
    """The bound changes nothing for FP64 factors, nor for BK pivoting (its
    2x2 pivots have a ratio above 0.42)."""
    rp, ci, v, bs, ip = planted_pairs(seed=3)
    S64 = oracle.Sym(rp, ci, bs, 0, 1.0)
    a = S64.factor(v, is_piv=ip, pivot=cb.PIV_STATIC).export()
    b = S64.factor(v, is_piv=ip, pivot=cb.PIV_STATIC, pivot_fp64=0.0).export()
    assert np.array_equal(a["val"], b["val"]) and np.array_equal(a["tri"], b["tri"])
    from problems import scrambled_kkt

    rp, ci, v, bs = scrambled_kkt(seed=11)
    S32 = oracle.Sym(rp, ci, bs, 0, 1.0, dtype=np.float32)
    a = S32.factor(v.astype(np.float32), pivot=cb.PIV_BK).export()
    b = S32.factor(v.astype(np.float32), pivot=cb.PIV_BK, pivot_fp64=0.0).export()
    assert (a["is_piv"] == 0).any()  # 2x2 pivots present
    assert np.array_equal(a["val"], b["val"]) and np.array_equal(a["tri"], b["tri"])


@pytest.mark.gpu
@pytest.mark.parametrize("bound", [1e-3, 0.0])
def test_gpu_fp64_inversion_matches_oracle(bound):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rp, ci, v, bs, ip = planted_pairs()
    n = len(rp) - 1
    h = cb.Handle(0)
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F32)
    F = cb.Factor(P)
    F.set_pivot_fp64(bound)
    F.compute(torch.from_numpy(v.astype(np.float32)).cuda(), is_piv=ip, pivot=cb.PIV_STATIC)
    OF = oracle.Sym(rp, ci, bs, 0, 1.0, dtype=np.float32).factor(v.astype(np.float32), is_piv=ip,
                                                                  pivot=cb.PIV_STATIC, pivot_fp64=bound)
    E, Eo = F.export(), OF.export()
    for k in ("blk_off", "idx", "val", "tri", "is_piv", "perm"):
        assert np.array_equal(E[k], Eo[k]), k
    b = cb.normal_vector(cb.SEED + 3, n).astype(np.float32)
    for stage in (cb.LEFT, cb.MIDDLE, cb.RIGHT):
        y = F.apply(stage, torch.from_numpy(b).cuda()).cpu().numpy()
        assert np.array_equal(y, OF.apply(stage, b)), stage


@pytest.mark.gpu
def test_gpu_fp32_static_pairs_match_reference_without_bound():
    """bound 0 is the reference's float arithmetic: the reference's own FP32
    factor of the planted problem, bit for bit; its error against the FP64
    factor is the one the FP64 inversion removes."""
    torch = pytest.importorskip("torch")
    from oracle import ref

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not ref.available():
        pytest.skip("reference build (oracle/_ref) not present")
    rp, ci, v, bs, ip = planted_pairs()
    n = len(rp) - 1
    b = cb.normal_vector(cb.SEED + 1, n)
    R = ref.run(rp, ci, v, bs, b, is_piv=ip, precision=0, pivot=cb.PIV_STATIC, max_it=0)
    theirs = ref.canonical_blocks(R)
    h = cb.Handle(0)
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F32)
    F = cb.Factor(P)
    F.set_pivot_fp64(0.0)
    F.compute(torch.from_numpy(v.astype(np.float32)).cuda(), is_piv=ip, pivot=cb.PIV_STATIC)
    pe = P.export()
    rows = np.repeat(np.arange(len(pe["coarse_off"]) - 1), np.diff(pe["coarse_off"]))
    mine = ref.canonical_export(F.export(), rows, pe["coarse_col"], pe["fmt"])
    assert set(mine) == set(theirs)
    for key, (fr, nr, _gr, ir, vr) in theirs.items():
        fm, nm, _gm, im, vm = mine[key]
        assert fm == fr and np.array_equal(im, ir) and np.array_equal(vm, vr), key
    E = F.export()
    for k in ("tri", "is_piv", "perm"):
        assert np.array_equal(E[k], R[k]), k
    y = F.apply(cb.MIDDLE, torch.from_numpy(b.astype(np.float32)).cuda()).cpu().numpy()
    assert np.array_equal(y, R["apply_middle"])
    E64 = oracle.Sym(rp, ci, bs, 0, 1.0).factor(v, is_piv=ip, pivot=cb.PIV_STATIC).export()
    F.set_pivot_fp64(1e-3)
    F.compute(torch.from_numpy(v.astype(np.float32)).cuda(), is_piv=ip, pivot=cb.PIV_STATIC)
    assert _factor_err(E, E64) > 1e-2 and _factor_err(F.export(), E64) < 1e-6
