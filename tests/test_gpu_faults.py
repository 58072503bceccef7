"""Failure paths made on the host, none of which faults the GPU: device
allocations that fail (injected with fk20_test_fail_allocations, as if the
device were full), requests that fail validation, and requests cancelled
before they reach the GPU.  Each must report its error code, leave the
context or server usable, and leave every other result exact."""
import ctypes
import time

import numpy as np
import pytest

import oracle as O
from conftest import fk20_setup_data

pytestmark = pytest.mark.gpu


def test_injected_allocation_failures_report_enomem_and_recover(engine):
    import torch
    n, rows, m = 1024, 40, 128
    xext = engine.to_device(fk20_setup_data(n)[2])
    poly = engine.to_device(O.seeded_fr(8080, rows * n).reshape(rows, n, 4))
    lib = engine.lib()
    c = engine.Context(0, 8)
    try:
        # the table build fails, then succeeds once the injection is spent
        assert lib.fk20_test_fail_allocations(1) == 0
        with pytest.raises(engine.Fk20Error) as err:
            c.load_xext_fft(n, xext)
        assert err.value.code == engine.FK20_ENOMEM
        c.load_xext_fft(n, xext)
        # the first pipeline call grows the workspace: it fails, the next one works
        h = engine.empty((rows, m, 18))
        assert lib.fk20_test_fail_allocations(1) == 0
        with pytest.raises(engine.Fk20Error) as err:
            c.poly2h_fft(h, poly, rows, n)
        assert err.value.code == engine.FK20_ENOMEM
        c.poly2h_fft(h, poly, rows, n)
        torch.cuda.synchronize()
        assert c.status() == 0
        got = O.g1_normalize(engine.to_host(h).reshape(-1, 18)).reshape(rows, m, 18)
        exp = O.fk20_rows(O.seeded_fr(8080, rows * n).reshape(rows, n, 4)[:2], fk20_setup_data(n)[2])
        assert np.array_equal(got[:2], exp)
        # a server whose slot buffers cannot be allocated is not created
        assert lib.fk20_test_fail_allocations(1) == 0
        with pytest.raises(engine.Fk20Error) as err:
            engine.Server(c, max_rows=8, slots=1)
        assert err.value.code == engine.FK20_ENOMEM
    finally:
        lib.fk20_test_fail_allocations(0)
        c.close()


@pytest.fixture(scope="module")
def ctx1024(engine):
    c = engine.Context(0, 8)
    c.load_xext_fft(1024, engine.to_device(fk20_setup_data(1024)[2]))
    yield c
    c.close()


def test_poisoned_requests_fail_validation(engine, ctx1024):
    """A request with an unsupported length, a null buffer, or a length whose
    tables are not loaded is refused at submit; the server keeps serving."""
    lib = engine.lib()
    srv = engine.Server(ctx1024, max_rows=8, slots=1)
    try:
        poly = O.seeded_fr(81, 1024)
        out = np.zeros((128, 18), np.uint64)
        t = ctypes.c_uint64()
        P = lambda a: ctypes.c_void_p(a.ctypes.data)
        assert lib.fk20_server_submit(srv.h, P(poly), 1000, P(out), ctypes.byref(t)) == engine.FK20_EINVAL
        assert lib.fk20_server_submit(srv.h, None, 1024, P(out), ctypes.byref(t)) == engine.FK20_EINVAL
        big = O.seeded_fr(82, 4096)
        assert lib.fk20_server_submit(srv.h, P(big), 4096, P(np.zeros((512, 18), np.uint64)),
                                      ctypes.byref(t)) == engine.FK20_ENOSETUP
        ticket = srv.submit(poly, out)
        assert srv.wait(ticket, 60000) == 0
        h = engine.empty((1, 128, 18))
        ctx1024.poly2h_fft(h, engine.to_device(poly.reshape(1, 1024, 4)), 1, 1024)
        assert np.array_equal(engine.to_host(h)[0], out)
    finally:
        srv.close()


def test_cancel_before_packing(engine, ctx1024):
    """With one slot and one request per pack, later submissions wait in the
    queue; cancelling them frees their buffers at once and their wait reports
    FK20_ECANCELED; a request already on the GPU cannot be cancelled
    (FK20_EAGAIN) and completes; every completed result is exact."""
    srv = engine.Server(ctx1024, max_rows=1, slots=1)
    try:
        polys = [O.seeded_fr(900 + j, 1024) for j in range(8)]
        outs = [np.zeros((128, 18), np.uint64) for _ in polys]
        tickets = [srv.submit(polys[j], outs[j]) for j in range(8)]
        rcs = {j: srv.cancel(tickets[j]) for j in (7, 6, 5, 0)}
        assert rcs[7] == 0 and rcs[6] == 0 and rcs[5] == 0  # queued behind a one-request slot
        assert rcs[0] in (0, engine.FK20_EAGAIN)
        cancelled = [j for j, rc in rcs.items() if rc == 0]
        deadline = time.time() + 120
        for j, t in enumerate(tickets):
            rc = srv.wait(t, max(1, int(1000 * (deadline - time.time()))))
            assert rc == (engine.FK20_ECANCELED if j in cancelled else 0), j
        st = srv.stats()
        assert st["cancelled"] == len(cancelled)
        assert srv.cancel(tickets[1]) == engine.FK20_EINVAL  # finished and waited for
        for j in range(8):
            if j in cancelled:
                continue
            h = engine.empty((1, 128, 18))
            ctx1024.poly2h_fft(h, engine.to_device(polys[j].reshape(1, 1024, 4)), 1, 1024)
            assert np.array_equal(engine.to_host(h)[0], outs[j]), j
    finally:
        srv.close()
