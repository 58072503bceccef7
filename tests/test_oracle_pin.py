"""The oracle reproduces the golden FK20 vectors produced by the reference's
own CUDA kernels on a B200 (tests/golden/reference_fk20_pin.json, written by
tests/golden/make_ref_gpu_fixtures.py)."""
import json
import os

import numpy as np
import pytest

import oracle as O
from conftest import ROOT

PIN = os.path.join(ROOT, "tests", "golden", "reference_fk20_pin.json")


@pytest.mark.skipif(not os.path.exists(PIN), reason="reference FK20 pin not generated yet")
def test_oracle_matches_reference_kernel_vectors():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_ref_gpu_fixtures as G
    pin = json.load(open(PIN))
    inp = pin["inputs"]
    tau = O.seeded_fr(inp["tau_seed"], 1)[0]
    setup = O.setup(tau, inp["n"] + 1)
    xext = O.xext_fft(setup, inp["n"], inp["l"])
    assert G.digest(xext) == inp["xext_fft_sha256"]
    poly = O.seeded_fr(inp["poly_seed"], inp["rows"] * inp["n"]).reshape(inp["rows"], inp["n"], 4)
    for r in range(inp["rows"]):
        res = O.fk20_row(poly[r], xext)
        for k in ("tc", "tc_fft", "hext_fft", "h", "h_fft"):
            assert G.digest(res[k]) == pin["sha256"][k][r], (k, r)
    # a mangled expectation must not match (reference NEGCMPCHECK pattern, test.h:116-122)
    res0 = O.fk20_row(poly[0], xext)["h_fft"].copy()
    res0[5, 0] ^= np.uint64(1)
    assert G.digest(res0) != pin["sha256"]["h_fft"][0]
