"""The C++ host program fk20-cuda_b200/host/fk20_prove drives the library
through the C ABI alone (fk20_ctx_create, fk20_ctx_load_setup,
fk20_ctx_poly2h_fft / fk20_ctx_poly2proofs): from files of setup points and
polynomials it writes the same proofs as the oracle, as h_fft and in the
data-availability format (FK20Py/fk20_multi.py:107-118)."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, fk20_setup_data

TOOL = os.path.join(ROOT, "fk20-cuda_b200", "host", "fk20_prove")


@pytest.mark.gpu
def test_host_program_matches_the_oracle(engine, tmp_path):
    assert os.access(TOOL, os.X_OK), "build the library first (make -C fk20-cuda_b200)"
    n, rows = 1024, 3
    tau, setup, xext = fk20_setup_data(n)
    polys = O.seeded_fr(7700, rows * n).reshape(rows, n, 4)
    sp, pp = tmp_path / "setup.bin", tmp_path / "poly.bin"
    sp.write_bytes(np.ascontiguousarray(setup[:n]).tobytes())
    pp.write_bytes(np.ascontiguousarray(polys).tobytes())
    out, out_da = tmp_path / "h_fft.bin", tmp_path / "da.bin"
    for target, extra in ((out, []), (out_da, ["--da"])):
        r = subprocess.run([TOOL, str(n), str(rows), str(sp), str(pp), str(target)] + extra, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr
    m = n // 8
    h = np.frombuffer(out.read_bytes(), np.uint64).reshape(rows, m, 18)
    exp = np.stack([O.fk20_row(polys[i], xext)["h_fft"] for i in range(rows)])
    assert np.array_equal(O.g1_normalize(h), exp)
    da = np.frombuffer(out_da.read_bytes(), np.uint8).reshape(rows, m, 48)
    assert np.array_equal(da, O.da_proofs(exp))


def test_host_program_reports_errors(tmp_path):
    """A wrong length or a short input file: a message and exit status 1
    (checked before any CUDA call, so no GPU is needed)."""
    assert os.access(TOOL, os.X_OK)
    p = tmp_path / "x.bin"
    p.write_bytes(b"\0" * 64)
    r = subprocess.run([TOOL, "1000", "1", str(p), str(p), str(tmp_path / "o.bin")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 1 and "n must be" in r.stderr
    r = subprocess.run([TOOL, "1024", "1", str(p), str(p), str(tmp_path / "o.bin")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 1 and "reading" in r.stderr
