"""KZG commitments (commit_to_poly, FK20Py/kzg_proofs.py:159-163): the
fixed-base MSM over the setup gives sum_i poly_i * s_i, checked against the
oracle's explicit linear combination and, at full size, against [f(tau)] G1
(the setup is tau^i G1 with tau known)."""
import numpy as np
import pytest

import oracle as O
from conftest import fk20_setup_data

pytestmark = pytest.mark.gpu


def test_commitments(engine):
    n, rows = 4096, 37
    tau, setup, _ = fk20_setup_data(n)
    c = engine.Context(0)
    c.load_commit(n, engine.to_device(setup[:n]), 9)
    poly = O.seeded_fr(3100, rows * n).reshape(rows, n, 4)
    poly[5] = 0  # zero polynomial -> infinity
    out = engine.empty((rows, 18))
    c.commit(out, engine.to_device(poly), rows, n)
    got = O.g1_normalize(engine.to_host(out))
    t = O.limbs_to_int(tau)
    g = O.g1_generator().reshape(1, 18)
    for r in (0, 5, 17, rows - 1):
        f_tau = 0
        for i in reversed(range(n)):
            f_tau = (f_tau * t + O.limbs_to_int(poly[r, i])) % O.R
        exp = O.g1_op("mul", g, O.int_to_limbs(f_tau, 4).reshape(1, 4))
        assert np.array_equal(got[r], exp[0]), r
    # a shorter polynomial against the explicit linear combination, with
    # non-canonical coefficients (x + r) that must not change the result
    k, short = 64, O.seeded_fr(3200, 2 * 64).reshape(2, 64, 4)
    nc = short.copy()
    for i in range(0, k, 5):
        v = O.limbs_to_int(nc[1, i]) + O.R
        if v < 1 << 256:
            nc[1, i] = O.int_to_limbs(v, 4)
    out2 = engine.empty((2, 18))
    c.commit(out2, engine.to_device(nc), 2, k)
    got2 = O.g1_normalize(engine.to_host(out2))
    for r in range(2):
        terms = O.g1_op("mul", setup[:k], short[r])
        acc = terms[0:1]
        for i in range(1, k):
            acc = O.g1_op("add", acc, terms[i:i + 1])
        assert np.array_equal(got2[r], O.g1_normalize(acc)[0])
    with pytest.raises(engine.Fk20Error) as e:
        c.commit(out2, engine.to_device(nc), 2, 40)  # not a multiple of 32
    assert e.value.code == engine.FK20_EINVAL
    c.close()
