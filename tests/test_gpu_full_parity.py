"""Every proof of the headline batch against the reference's own CUDA kernels.

512 rows x 4096 coefficients (262,144 proofs), seeded, one shared setup: the
reference's host pipeline fk20_poly2h_fft (fk20_poly2h_fft.cu:47-78, the
reference library compiled unmodified for sm_100a into oracle/_ref by
oracle/ref/Makefile) and this library's C-ABI fk20_poly2h_fft run on the same
device buffers, and every output point is compared on the GPU by projective
equality (g1p_eq_n), which is equality after affine normalisation.  Two rows
are also checked against the oracle, so the comparison does not rest on the
two GPU paths alone.  This is the reference's own full-size test
(fk20_512test.cu:139-263, fullTest_512) with seeded inputs in place of its
missing test-vector file."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, fk20_setup_data

pytestmark = pytest.mark.gpu
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libfk20ref.so")


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference library not built (oracle/ref/Makefile)")
def test_all_262144_proofs_equal_reference_kernels(engine):
    import torch
    n, rows, m = 4096, 512, 512
    _, _, xext = fk20_setup_data(n)
    poly = O.seeded_fr(2024, rows * n).reshape(rows, n, 4)
    poly[5] = 0                              # a zero row: all proofs at infinity
    poly[6] = 0
    poly[6, 4095] = O.int_to_limbs(1, 4)     # one non-zero coefficient
    poly[7, :] = O.int_to_limbs(O.R - 1, 4)  # the largest canonical value everywhere
    dpoly = engine.to_device(poly)
    dxext = engine.to_device(xext)
    ref_out = engine.empty((rows, m, 18))
    ours = engine.empty((rows, m, 18))
    lib = ctypes.CDLL(REF_LIB, mode=os.RTLD_LOCAL)
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    torch.cuda.synchronize()
    assert lib.ref_fk20_poly2h_fft(P(ref_out), P(dpoly), P(dxext), ctypes.c_uint(rows)) == 0
    engine.call("fk20_poly2h_fft", engine._ptr(ours), engine._ptr(dpoly), engine._ptr(dxext), rows)
    eq = torch.zeros(rows * m, dtype=torch.uint8, device="cuda")
    engine.call("g1p_eq_n", engine._ptr(eq), engine._ptr(ours), engine._ptr(ref_out), rows * m, engine._stream())
    torch.cuda.synchronize()
    bad = torch.nonzero(eq == 0).flatten().cpu().numpy()
    assert bad.size == 0, f"{bad.size} of {rows * m} proofs differ, first at (row, proof) {divmod(int(bad[0]), m)}"
    # the reference's zero row is all infinity, and the two paths agree with the oracle on two rows
    h = O.g1_normalize(engine.to_host(ours).reshape(-1, 18)).reshape(rows, m, 18)
    assert np.all(h[5, :, 12:] == 0)
    exp = O.fk20_rows(poly[[6, 300]], xext)
    assert np.array_equal(h[6], exp[0]) and np.array_equal(h[300], exp[1])
