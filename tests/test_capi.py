"""The C-ABI library loads (no GPU needed) and exports every symbol that
include/culipx.h declares; host-only entry points work without a device."""
import ctypes
import os
import re

import numpy as np

import culip_b200 as cb
from culip_b200 import _capi as capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "culipx.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(culipx_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = capi.load()
    names = _declared()
    assert len(names) >= 25
    for name in names:
        assert hasattr(L, name), name
    # every declared symbol has a binding with a signature
    for name in names:
        assert name in capi.declared_symbols(), name


def test_version_and_error_string():
    L = capi.load()
    assert L.culipx_version() >= 10000
    st = L.culipx_kkt_nnz(None, None)
    assert st == capi.INVALID_ARG
    assert b"culipx_kkt_nnz" in L.culipx_last_error()


def test_host_only_handle_rejects_device_work():
    h = ctypes.c_void_p()
    capi.call("culipx_handle_create", ctypes.byref(h), -1, None)
    rp, ci, v = cb.kkt_generate(40, 20, 2, 0, 1, 10)
    bs = cb.kkt_blocking(40, 20, 4)
    p = ctypes.c_void_p()
    capi.call("culipx_pattern_analyze", h, 60, rp.ctypes.data_as(ctypes.c_void_p), ci.ctypes.data_as(ctypes.c_void_p),
              len(bs) - 1, bs.ctypes.data_as(ctypes.c_void_p), 0, 1.0, cb.F64, ctypes.byref(p))
    f = ctypes.c_void_p()
    assert capi.load().culipx_factor_create(p, ctypes.byref(f)) == capi.INVALID_ARG
    capi.load().culipx_pattern_destroy(p)
    capi.load().culipx_handle_destroy(h)


def test_normal_vector_deterministic():
    a = cb.normal_vector(5, 1001)
    b = cb.normal_vector(5, 1001)
    assert np.array_equal(a, b)
    assert abs(a.mean()) < 0.15 and abs(a.std() - 1) < 0.1
