"""chains.inc (the one-statement PTX carry chains of the Fp / Fr arithmetic)
is what gen_chains.py writes: the generator re-run here must reproduce the
committed file."""
import os
import subprocess
import sys

from conftest import ROOT

CSRC = os.path.join(ROOT, "fk20-cuda_b200", "csrc")


def test_chains_are_the_generators_output():
    out = subprocess.run([sys.executable, "gen_chains.py"], cwd=CSRC, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    with open(os.path.join(CSRC, "chains.inc")) as f:
        assert out.stdout == f.read()
