"""The imported L D L' preconditioner on the reference's own SQMR fixtures
(tests/la/test_sqmr.cc:192-293): its three applies equal the restatement's
bit for bit, and SQMR with it meets the reference test's assertions."""
import numpy as np
import pytest
import scipy.sparse as sp

import culip_b200 as cb
import oracle
from test_oracle_golden import _load, tridiag_from_D

pytestmark = pytest.mark.gpu


def _fixture(case):
    d = _load(f"sqmr_{case}.npz")
    n = len(d["A_rowptr"]) - 1
    tri, is_piv = tridiag_from_D(d["D_rowptr"], d["D_colidx"], d["D_val"], n)
    return d, n, tri, is_piv


def _ldu(h, d, tri, is_piv):
    import torch

    t = lambda a, dt: torch.from_numpy(np.ascontiguousarray(a, dt)).cuda()
    return cb.ImportLDU(h, t(d["L_rowptr"], np.int32), t(d["L_colidx"], np.int32), t(d["L_val"], np.float64),
                        t(tri, np.float64), t(is_piv, np.int32), t(d["perm"], np.int32), t(d["scale"], np.float64))


@pytest.mark.parametrize("case", ["small", "big"])
@pytest.mark.parametrize("stage", [cb.LEFT, cb.MIDDLE, cb.RIGHT])
def test_ldu_apply_bit_exact(case, stage):
    import torch

    h = cb.Handle(0)
    d, n, tri, is_piv = _fixture(case)
    P = _ldu(h, d, tri, is_piv)
    b = cb.normal_vector(31, n)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    P.apply(stage, torch.from_numpy(b).cuda(), x)
    ref = oracle.ldu_apply(d["L_rowptr"], d["L_colidx"], d["L_val"], tri, is_piv, d["perm"], d["scale"], stage, b)
    assert np.array_equal(x.cpu().numpy(), ref)


@pytest.mark.parametrize("case", ["small", "big"])
def test_sqmr_ldu_reference_fixture(case):
    import torch

    h = cb.Handle(0)
    d, n, tri, is_piv = _fixture(case)
    rp, ci, v = d["A_rowptr"], d["A_colidx"], d["A_val"]
    A = sp.csr_matrix((v, ci, rp), shape=(n, n))
    b = A @ np.ones(n)
    P = _ldu(h, d, tri, is_piv)
    Ag = cb.CsrOperator(h, torch.from_numpy(np.ascontiguousarray(rp, np.int32)).cuda(),
                        torch.from_numpy(np.ascontiguousarray(ci, np.int32)).cuda(), torch.from_numpy(v).cuda())
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    res, its, st = P.sqmr_solve(Ag, torch.from_numpy(b).cuda(), x, 1e-10, n)
    x = x.cpu().numpy()
    # the reference test's assertions (term_tol 1e-10, test_tol 1e-5, iterations <= n)
    assert np.linalg.norm(b - A @ x) <= 1e-5 * np.linalg.norm(b)
    assert its <= n
    xo, reso, ito = oracle.sqmr_ldu(rp, ci, v, d["L_rowptr"], d["L_colidx"], d["L_val"], tri, is_piv, d["perm"],
                                    d["scale"], b, 1e-10, n)
    assert abs(its - ito) <= 4
