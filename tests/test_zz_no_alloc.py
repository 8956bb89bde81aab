"""culipx_sqmr_solve_noalloc: the SQMR solve for callers that cannot allocate
device memory while they solve (GPU memory already owned by another
allocator, or request loops where cudaMalloc / cudaFree could synchronize the
device).  It must give the regular entry point's results, call after call,
from the fixed scratch compiled into the library.

Collected last on purpose (file name), so a run that stops at the first
failure has run every other test first; it also passes alone in a fresh
process (the first call does the per-device scratch set-up).
"""
import numpy as np
import pytest

import culip_b200 as cb
from problems import kkt

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def setup():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    h = cb.Handle(0)
    rp, ci, v, bs = kkt("small")
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F64)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v).cuda())
    A = cb.CsrOperator(h, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    b = torch.from_numpy(cb.normal_vector(cb.SEED + 1, len(rp) - 1)).cuda()
    return h, A, F, b, len(rp) - 1


def test_noalloc_matches_regular_entry_point_twice(setup):
    h, A, F, b, n = setup
    x_ref = torch.zeros(n, dtype=torch.float64, device="cuda")
    res_ref, its_ref, st_ref = cb.sqmr_solve(h, A, F, b, x_ref, 1e-8, 1000)
    xr = x_ref.cpu().numpy()
    for _ in range(2):  # two calls in a row: the shared scratch keeps the previous call's contents
        x = torch.full((n,), 7.0, dtype=torch.float64, device="cuda")
        res, its, st = cb.sqmr_solve_noalloc(h, A, F, b, x, 1e-8, 1000)
        xn = x.cpu().numpy()
        assert st == st_ref
        assert abs(its - its_ref) <= 4
        assert np.linalg.norm(xn - xr) / np.linalg.norm(xr) < 1e-6
        assert abs(res - res_ref) <= 1e-6 * max(abs(res_ref), 1e-30) + 1e-14


def test_noalloc_rejects_sizes_beyond_its_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    h = cb.Handle(0)
    n = 70000  # > 65536 rows of fixed scratch
    rp, ci, v = cb.kkt_generate(n - 20000, 20000, 2, 0, 1, 10)
    bs = cb.kkt_blocking(n - 20000, 20000, 32)
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, cb.F64)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v).cuda())
    A = cb.CsrOperator(h, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    b = torch.ones(n, dtype=torch.float64, device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(cb.CulipxError) as e:
        cb.sqmr_solve_noalloc(h, A, F, b, x, 1e-8, 10)
    assert "65536" in str(e.value)
