"""pairing_consts.inc is what gen_pairing_consts.py writes: the generator
re-run here must reproduce the committed file, and in doing so re-checks its
assertions (the decomposition of the final exponent that kernels_pairing.cu
computes, 3 (p^4 - p^2 + 1)/r = (z - 1)^2 (z + p)(z^2 + p^2 - 1) + 3, and the
32nd root of unity of Fr)."""
import os
import subprocess
import sys

from conftest import ROOT

CSRC = os.path.join(ROOT, "fk20-cuda_b200", "csrc")


def test_pairing_constants_are_the_generators_output():
    out = subprocess.run([sys.executable, "gen_pairing_consts.py"], cwd=CSRC, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr
    with open(os.path.join(CSRC, "pairing_consts.inc")) as f:
        assert out.stdout == f.read()
