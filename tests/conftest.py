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


def kzg_multi_case(l=4, deg=8, tau=0x5EED5EED1234567, seed=77):
    """A small check_proof_multi case built from the KZG definitions, with tau
    known: f, x, ys[k] = f(x w^k), the commitment [f(tau)]G1 and the proof
    [q(tau)]G1, q = (f - I) / (X^l - x^l), I = f mod (X^l - x^l)."""
    import random
    import oracle as O
    import pairing_py as PP
    rnd = random.Random(seed)
    R = O.R
    f = [rnd.randrange(R) for _ in range(deg)]
    x = rnd.randrange(1, R)
    w = pow(5, (R - 1) // l, R)
    ev = lambda z: sum(c * pow(z, i, R) for i, c in enumerate(f)) % R
    ys = [ev(x * pow(w, k, R) % R) for k in range(l)]
    xl = pow(x, l, R)
    rem = [sum(f[k + l * q] * pow(xl, q, R) for q in range((deg - k + l - 1) // l)) % R for k in range(l)]
    i_tau = sum(c * pow(tau, k, R) for k, c in enumerate(rem)) % R
    q_tau = (ev(tau) - i_tau) * pow((pow(tau, l, R) - xl) % R, R - 2, R) % R
    g = O.g1_generator()
    G1 = (O.limbs_to_int(g[0:6]), O.limbs_to_int(g[6:12]))
    G2 = PP.g2_generator()
    return dict(f=f, x=x, ys=ys, tau=tau, commitment=PP.g1mul(ev(tau), G1), proof=PP.g1mul(q_tau, G1),
                setup_g1=[PP.g1mul(pow(tau, k, R), G1) for k in range(l)],
                setup_g2=[PP.g2mul(pow(tau, k, R), G2) for k in range(l + 1)])
