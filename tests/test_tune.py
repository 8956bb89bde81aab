"""The KKT block-size tuner: it times every candidate's factor + solve and
returns the fastest candidate that met the tolerance (else the one whose
solve got furthest)."""
import numpy as np
import pytest

import culip_b200 as cb
from culip_b200 import _capi as capi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [cb.F32, cb.F64])
def test_tune_kkt_block(precision):
    import torch

    h = cb.Handle(0)
    n, m = 3000, 1500
    rp, ci, v = cb.kkt_generate(n, m, 6, 32, 1e-2, 1e2, seed=cb.SEED + 77)
    b = cb.normal_vector(cb.SEED + 78, n + m)
    best, res = cb.tune_kkt_block(h, n, m, rp, ci, torch.from_numpy(v).cuda(), torch.from_numpy(b).cuda(),
                                  precision, (8, 16, 32), 1e-8, 1000)
    assert best in (8, 16, 32) and set(res) == {8, 16, 32}
    for ms, its, st, rr in res.values():
        assert ms > 0 and 0 < its <= 1000 and st in (capi.OK, capi.MAXIT, capi.BREAKDOWN)
    ok = {c: r for c, r in res.items() if r[2] == capi.OK}
    if ok:
        assert res[best][2] == capi.OK and res[best][0] == min(r[0] for r in ok.values())
    else:
        assert res[best][3] == min(r[3] for r in res.values())
    # the tuned blocking is a valid pattern for the solver
    bs = cb.kkt_blocking(n, m, best)
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, precision)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v.astype(np.float32 if precision == cb.F32 else np.float64)).cuda())
    A = cb.CsrOperator(h, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    x = torch.zeros(n + m, dtype=torch.float64, device="cuda")
    r, its, st = cb.sqmr_solve(h, A, F, torch.from_numpy(b).cuda(), x, 1e-8, 1000)
    assert its == res[best][1]
