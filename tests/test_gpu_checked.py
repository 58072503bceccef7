"""The checked build (libfk20b200_checked.so, `make -C fk20-cuda_b200 checked`;
csrc/check.cuh): the same kernels with their index and range checks
compiled in.  It must give the normal build's results, report no failure on
valid work, and report -- without trapping -- a failure planted through the
test hook FK20_OPT_TEST_CHECK (a flag nothing else sets), after which the
next call is clean.  The normal build reports that nothing is compiled in."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, fk20_setup_data

pytestmark = pytest.mark.gpu
PKG = os.path.join(ROOT, "fk20-cuda_b200")


@pytest.fixture(scope="module")
def checked(engine):
    path = os.path.join(PKG, "libfk20b200_checked.so")
    if not os.path.exists(path):
        subprocess.run(["make", "-s", "-j8", "-C", PKG, "checked"], check=True)
    L = ctypes.CDLL(path)
    vp, u, i = ctypes.c_void_p, ctypes.c_uint, ctypes.c_int
    for name, args in {"fk20_ctx_create": [ctypes.POINTER(vp), i, i], "fk20_ctx_destroy": [vp],
                       "fk20_ctx_load_xext_fft": [vp, u, vp, vp], "fk20_ctx_poly2h_fft": [vp, vp, vp, u, u, vp],
                       "fk20_ctx_set": [vp, i, i], "fk20_ctx_status": [vp],
                       "fk20_check_status": [ctypes.POINTER(i)]}.items():
        getattr(L, name).argtypes = args
        getattr(L, name).restype = i
    return L


def status(L):
    c = ctypes.c_int(-1)
    rc = L.fk20_check_status(ctypes.byref(c))
    return rc, c.value


def test_normal_build_has_no_checks(engine):
    assert status(engine.lib()) == (0, 0)


def test_checked_build_agrees_and_reports_planted_failure(engine, checked):
    import torch
    n, rows, m = 1024, 33, 128
    _, _, xext = fk20_setup_data(n)
    dx = engine.to_device(xext)
    poly = engine.to_device(O.seeded_fr(4711, rows * n).reshape(rows, n, 4))
    ref = engine.empty((rows, m, 18))
    c0 = engine.Context(0, 8)
    c0.load_xext_fft(n, dx)
    c0.poly2h_fft(ref, poly, rows, n)
    torch.cuda.synchronize()
    c0.close()
    P = engine._ptr
    h = ctypes.c_void_p()
    assert checked.fk20_ctx_create(ctypes.byref(h), 0, 8) == 0
    try:
        assert checked.fk20_ctx_load_xext_fft(h, n, P(dx), None) == 0
        out = engine.empty((rows, m, 18))
        assert checked.fk20_ctx_poly2h_fft(h, P(out), P(poly), rows, n, None) == 0
        assert checked.fk20_ctx_status(h) == 0
        assert status(checked) == (0, 1)
        assert torch.equal(out, ref)
        # planted: the MSM records FK20_CHECK_MSM_PLANTED; the status is taken once
        assert checked.fk20_ctx_set(h, engine.FK20_OPT_TEST_CHECK, 1) == 0
        assert checked.fk20_ctx_poly2h_fft(h, P(out), P(poly), rows, n, None) == 0
        assert status(checked) == (3, 1)
        assert status(checked) == (0, 1)
        assert checked.fk20_ctx_set(h, engine.FK20_OPT_TEST_CHECK, 0) == 0
        out2 = engine.empty((rows, m, 18))
        assert checked.fk20_ctx_poly2h_fft(h, P(out2), P(poly), rows, n, None) == 0
        assert checked.fk20_ctx_status(h) == 0 and status(checked) == (0, 1)
        assert torch.equal(out2, ref)
    finally:
        checked.fk20_ctx_destroy(h)
