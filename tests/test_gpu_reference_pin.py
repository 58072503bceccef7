"""Three-way parity on the GPU: the reference's own kernels (oracle/_ref,
compiled unmodified for sm_100a), the oracle and the engine agree on every
FK20 intermediate for the same seeded inputs."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, fk20_setup_data

pytestmark = pytest.mark.gpu
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libfk20ref.so")


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference library not built (oracle/ref/Makefile)")
def test_reference_kernels_oracle_engine_agree(engine):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_ref_gpu_fixtures as G
    n, rows = 4096, 3
    tau, setup, xext = fk20_setup_data(n)
    poly = O.seeded_fr(91, rows * n).reshape(rows, n, 4)
    poly[2] = 0
    poly[2, 7] = O.int_to_limbs(5, 4)
    ref = G.reference_run(poly, xext)
    ctx = engine.Context(0)
    ctx.load_xext_fft(n, engine.to_device(xext))
    h = engine.empty((rows, 512, 18))
    ctx.poly2h_fft(h, engine.to_device(poly), rows, n)
    ours = G.canon_g1(engine.to_host(h))
    for r in range(rows):
        exp = O.fk20_row(poly[r], xext)
        assert np.array_equal(G.canon_fr(ref["tc"][r]), exp["tc"])
        assert np.array_equal(G.canon_fr(ref["tc_fft"][r]), exp["tc_fft"])
        assert np.array_equal(G.canon_g1(ref["hext_fft"][r]), exp["hext_fft"])
        assert np.array_equal(G.canon_g1(ref["h"][r]), exp["h"])
        assert np.array_equal(G.canon_g1(ref["h_fft"][r]), exp["h_fft"])
        assert np.array_equal(ours[r], exp["h_fft"])
    ctx.close()
