"""Matrix-free KKT operators (AugmentedMatrixSPMV / NormalMatrixSPMV) against
the oracle's restatement, and the augmented product against the assembled K."""
import numpy as np
import pytest

import culip_b200 as cb
import oracle

pytestmark = pytest.mark.gpu


def _constraints(n, m, seed):
    rng = np.random.default_rng(seed)
    cols = [np.sort(rng.choice(n, int(rng.integers(1, 9)), replace=False)) for _ in range(m)]
    cols[3] = np.zeros(0, np.int64)  # an empty constraint row
    rp = np.concatenate([[0], np.cumsum([len(c) for c in cols])]).astype(np.int32)
    ci = np.concatenate(cols).astype(np.int32)
    return rp, ci, rng.standard_normal(len(ci)), 10.0 ** rng.uniform(-3, 3, n)


@pytest.mark.parametrize("kind", [cb.KktOperator.AUGMENTED, cb.KktOperator.NORMAL])
@pytest.mark.parametrize("shifted", [False, True])
def test_kkt_operator(kind, shifted):
    import torch

    h = cb.Handle(0)
    n, m = 700, 300
    rp, ci, v, d = _constraints(n, m, 3)
    ix = np.arange(0, m, 3, dtype=np.int32)[::-1].copy() if shifted else None
    delta = -1e-2 if shifted else 0.0
    t = lambda a: torch.from_numpy(a).cuda()
    op = cb.KktOperator(h, kind, m, n, t(rp), t(ci), t(v), t(d), delta, None if ix is None else t(ix))
    rows = n + m if kind == cb.KktOperator.AUGMENTED else m
    rng = np.random.default_rng(4)
    x = rng.standard_normal(rows)
    y0 = rng.standard_normal(rows)
    for alpha, beta in ((1.0, 0.0), (0.5, -2.0)):
        yg = t(y0.copy())
        op.multiply(t(x), yg, alpha, beta)
        ref = oracle.kkt_operator(kind, rp, ci, v, n, d, x, delta, ix, alpha, beta, y0)
        assert np.allclose(yg.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    if kind == cb.KktOperator.AUGMENTED:
        # the assembled K = [[D, A'], [A, shift]] gives the same product
        import scipy.sparse as sp

        A = sp.csr_matrix((v, ci, rp), shape=(m, n))
        shift = np.zeros(m)
        if ix is not None:
            shift[ix] = delta
        K = sp.bmat([[sp.diags(d), A.T], [A, sp.diags(shift)]]).tocsr()
        yg = t(np.zeros(rows))
        op.multiply(t(x), yg)
        assert np.allclose(yg.cpu().numpy(), K @ x, rtol=1e-12, atol=1e-12 * np.abs(K @ x).max())


def test_kkt_operator_rejects_bad_input():
    import torch

    h = cb.Handle(0)
    rp, ci, v, d = _constraints(50, 20, 5)
    ci_bad = ci.copy()
    ci_bad[0] = 50
    t = lambda a: torch.from_numpy(a).cuda()
    with pytest.raises(cb.CulipxError):
        cb.KktOperator(h, 0, 20, 50, t(rp), t(ci_bad), t(v), t(d))
    with pytest.raises(cb.CulipxError):
        cb.KktOperator(h, 1, 20, 50, t(rp), t(ci), t(v), t(d), 1.0, t(np.array([25], np.int32)))
