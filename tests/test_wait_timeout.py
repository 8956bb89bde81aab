"""The persistent solver's bounded device wait.

In the fused two-level iteration the level-0 rows wait on a device counter
for every CTA's level-1 rows instead of a grid barrier.  The wait is bounded
(200 ms): culipx_sqmr_set_wait_skew raises the count it waits for beyond
reach, so it gives up, the kernel finishes with its results marked invalid
and the solve returns CULIPX_TIMEOUT.  Nothing faults or hangs: the handle
stays usable and the next solve without the skew is the ordinary one, bit for
bit."""
import numpy as np
import pytest

import culip_b200 as cb
from culip_b200 import _capi as capi
from problems import kkt

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _system(h):
    rp, ci, v, bs = kkt("small")
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F64)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v).cuda())
    A = cb.CsrOperator(h, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    b = torch.from_numpy(cb.normal_vector(cb.SEED + 1, len(rp) - 1)).cuda()
    return P, F, A, b


def test_level_wait_times_out_and_the_handle_recovers():
    h = cb.Handle(0)
    P, F, A, b = _system(h)
    x_ref = torch.zeros_like(b)
    res_ref, its_ref, _ = cb.sqmr_solve(h, A, F, b, x_ref, 1e-8, 50)
    capi.call("culipx_sqmr_set_wait_skew", h._h, 1 << 40)
    x = torch.zeros_like(b)
    with pytest.raises(cb.CulipxError) as err:
        cb.sqmr_solve(h, A, F, b, x, 1e-8, 3)
    assert err.value.status == capi.TIMEOUT
    capi.call("culipx_sqmr_set_wait_skew", h._h, 0)
    x2 = torch.zeros_like(b)
    res2, its2, _ = cb.sqmr_solve(h, A, F, b, x2, 1e-8, 50)
    assert its2 == its_ref and res2 == res_ref
    assert torch.equal(x2, x_ref)


def test_level_wait_timeout_in_the_multi_rhs_solve():
    h = cb.Handle(0)
    P, F, A, b = _system(h)
    B = torch.stack([b, 2.0 * b])
    X = torch.zeros_like(B)
    capi.call("culipx_sqmr_set_wait_skew", h._h, 1 << 40)
    # the call succeeds; every right-hand side reports TIMEOUT
    res, its, st = cb.sqmr_solve_multi(h, A, F, B, X, 1e-8, 3)
    assert np.all(st == capi.TIMEOUT)
    capi.call("culipx_sqmr_set_wait_skew", h._h, 0)
    res, its, st = cb.sqmr_solve_multi(h, A, F, B, X, 1e-8, 20)
    assert np.all(st != capi.TIMEOUT)
