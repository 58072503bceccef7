import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", "fk20-cuda_b200", ""):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def kats():
    import json
    with open(os.path.join(ROOT, "tests", "golden", "reference_kats.json")) as f:
        return json.load(f)


_SETUP_CACHE = {}


def fk20_setup_data(n: int, seed: int = 424242):
    """(tau, setup[n+1], xext_fft[16][2n/16]) for polynomial length n, from the
    oracle (FK20Py/kzg_proofs.py:22-30, fk20_multi_cuda.py:104-109); cached."""
    key = (n, seed)
    if key not in _SETUP_CACHE:
        import oracle as O
        tau = O.seeded_fr(seed, 1)[0]
        setup = O.setup(tau, n + 1)
        xext = O.xext_fft(setup, n, 16)
        _SETUP_CACHE[key] = (tau, setup, xext)
    return _SETUP_CACHE[key]


@pytest.fixture(scope="session")
def engine():
    """The CUDA engine binding; GPU tests only."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    import fk20b200
    fk20b200.lib()
    return fk20b200
