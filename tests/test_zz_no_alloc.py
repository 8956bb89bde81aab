"""culipx_sqmr_solve_noalloc: the SQMR solve for callers that cannot allocate
device memory while they solve (GPU memory already owned by another
allocator, or request loops where cudaMalloc / cudaFree could synchronize the
device).  It runs the regular entry point's kernel with the regular grid and
reduction order from the fixed scratch compiled into the library, so its
results must equal the regular entry point's bit for bit, call after call.

Collected last on purpose (file name), so a run that stops at the first
failure has run every other test first; it also passes alone in a fresh
process (the first call does the per-device scratch set-up).
"""
import ctypes

import numpy as np
import pytest

import culip_b200 as cb
from culip_b200 import _capi as capi
from problems import kkt

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _system(prec):
    h = cb.Handle(0)
    rp, ci, v, bs = kkt("small")
    P = cb.Pattern(h, rp, ci, bs, 0, 1.0, prec)
    F = cb.Factor(P)
    F.compute(torch.from_numpy(v.astype(np.float32 if prec == cb.F32 else np.float64)).cuda())
    A = cb.CsrOperator(h, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(v).cuda())
    b = torch.from_numpy(cb.normal_vector(cb.SEED + 1, len(rp) - 1)).cuda()
    return h, A, F, b, len(rp) - 1


@pytest.mark.parametrize("prec", [cb.F64, cb.F32], ids=["f64_factor", "f32_factor"])
def test_noalloc_matches_regular_entry_point_twice(prec):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    # a fresh handle whose workspace the regular solve has not created yet:
    # the no-allocation calls below cannot borrow it
    h, A, F, b, n = _system(prec)
    outs = []
    for k in range(2):  # two calls in a row: the shared scratch keeps the previous call's contents
        x = torch.full((n,), 7.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        res, its, st = cb.sqmr_solve_noalloc(h, A, F, b, x, 1e-8, 1000)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        if k == 1:  # the first call may load the library's device module (the scratch lives in it)
            assert free1 == free0, f"device memory changed by {free0 - free1} bytes"
        outs.append((x.cpu().numpy(), res, its, st))
    x_ref = torch.zeros(n, dtype=torch.float64, device="cuda")
    res_ref, its_ref, st_ref = cb.sqmr_solve(h, A, F, b, x_ref, 1e-8, 1000)
    xr = x_ref.cpu().numpy()
    for xn, res, its, st in outs:
        assert st == st_ref and its == its_ref
        assert res == res_ref
        assert np.array_equal(xn, xr)


def test_noalloc_reports_maxit_without_an_iterations_pointer():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    h, A, F, b, n = _system(cb.F64)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    st = capi.call("culipx_sqmr_solve_noalloc", h._h, A._h, F._h, ctypes.c_void_p(b.data_ptr()),
                   ctypes.c_void_p(x.data_ptr()), 1e-14, 3, None, None, allow=(capi.OK, capi.MAXIT))
    assert st == capi.MAXIT


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
