"""The header-only device library include/fk20_device.cuh: the reference's
fp_* / fr_* / g1p_* device functions (fp.cuh:16-41, fr.cuh:33-58,
g1.cuh:31-96), called from kernels of a test probe (tests/host/devapi_probe.cu,
built by tests/host/Makefile), against the oracle -- standard-form values,
non-canonical inputs allowed, canonical outputs."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT

pytestmark = pytest.mark.gpu
HOST = os.path.join(ROOT, "tests", "host")


@pytest.fixture(scope="module")
def probe():
    subprocess.run(["make", "-s", "-C", HOST], check=True)  # no-op when the probe is current
    return ctypes.CDLL(os.path.join(HOST, "libdevapi_probe.so"))


def vals(rng, count, mod, limbs, noncanon=True):
    xs = [int.from_bytes(rng.bytes(8 * limbs), "little") % mod for _ in range(count)]
    xs[:4] = [0, 1, mod - 1, 2]
    if noncanon:  # any representative below 2^(64 limbs)
        for j in range(4, 12):
            if xs[j] + mod < 1 << (64 * limbs):
                xs[j] += mod
    return O.ints_to_array(xs, limbs)


def run(engine, fn, op, x, y, *extra):
    import torch
    dx, dy = engine.to_device(x), engine.to_device(y)
    dz = engine.empty(x.shape)
    dextra = [engine.to_device(e) for e in extra]
    assert fn(op, engine._ptr(dz), engine._ptr(dx), engine._ptr(dy), *[engine._ptr(e) for e in dextra],
              x.shape[0]) == 0
    torch.cuda.synchronize()
    return engine.to_host(dz)


def test_fp_device_api(engine, probe):
    rng = np.random.default_rng(41)
    x, y = vals(rng, 600, O.P, 6), vals(rng, 600, O.P, 6)[::-1].copy()
    exp = {0: O.fp_op("mul", x, y), 1: O.fp_op("sqr", x), 2: O.fp_op("add", x, y), 3: O.fp_op("sub", x, y),
           4: O.fp_op("neg", x), 6: O.fp_op("x3", x), 7: O.fp_op("x12", x), 9: O.fp_op("reduce", x)}
    for op, e in exp.items():
        assert np.array_equal(run(engine, probe.devapi_fp, op, x, y), e), op
    xi = x[:100]
    assert np.array_equal(run(engine, probe.devapi_fp, 5, xi, xi), O.fp_op("inv", xi))
    mma = O.fp_op("add", O.fp_op("mul", x, y), O.fp_op("sqr", y))
    assert np.array_equal(run(engine, probe.devapi_fp, 8, x, y), mma)
    eq = run(engine, probe.devapi_fp, 10, x, O.fp_op("reduce", x))  # x == canonical(x)
    assert np.all(eq[:, 0] == 1)


def test_fr_device_api(engine, probe):
    rng = np.random.default_rng(42)
    x, y = vals(rng, 600, O.R, 4), vals(rng, 600, O.R, 4)[::-1].copy()
    exp = {0: O.fr_op("mul", x, y), 1: O.fr_op("sqr", x), 2: O.fr_op("add", x, y), 3: O.fr_op("sub", x, y),
           4: O.fr_op("neg", x), 6: O.fr_op("x3", x), 7: O.fr_op("add", x, y), 8: O.fr_op("reduce", x)}
    for op, e in exp.items():
        assert np.array_equal(run(engine, probe.devapi_fr, op, x, y), e), op
    xi = x[:100]
    assert np.array_equal(run(engine, probe.devapi_fr, 5, xi, xi), O.fr_op("inv", xi))


def test_g1_device_api(engine, probe):
    rng = np.random.default_rng(43)
    g = O.g1_generator().reshape(1, 18)
    cnt = 96
    p = O.g1_op("mul", np.repeat(g, cnt, 0), O.seeded_fr(44, cnt))
    q = O.g1_op("mul", np.repeat(g, cnt, 0), O.seeded_fr(45, cnt))
    q[0] = p[0]                       # p + p through the addition law
    q[1] = O.g1_op("neg", p[1:2])[0]  # p + (-p) = infinity
    q[2] = 0
    q[2, 6:12] = [7, 0, 0, 0, 0, 0]   # infinity as (0, 7, 0)
    s = np.stack([O.int_to_limbs(int.from_bytes(rng.bytes(32), "little"), 4) for _ in range(cnt)])
    N = lambda a: O.g1_normalize(a)
    exp = {0: O.g1_op("add", p, q), 1: O.g1_op("dbl", p), 2: O.g1_op("sub", p, q), 3: O.g1_op("neg", p),
           4: O.g1_op("mul", p, s), 5: O.g1_op("dbl", p), 6: O.g1_op("add", p, q), 8: N(p)}
    for op, e in exp.items():
        got = run(engine, probe.devapi_g1, op, p, q, s)
        assert np.array_equal(N(got), N(e)), op
    flags = run(engine, probe.devapi_g1, 7, p, p, s)
    assert np.all(flags[:, 0] == 1) and np.all(flags[:, 6] == 1) and np.all(flags[:, 12] == 0)


def test_fp_mul_two_products_rate(engine, probe):
    """fp_mul costs two Montgomery products (MontMul then a product by R^2):
    same values as a convert-in / multiply / convert-out chain, and faster."""
    import torch
    n, iters = 1 << 20, 64
    rng = np.random.default_rng(46)
    x, y = vals(rng, n, O.P, 6, noncanon=False), vals(rng, n, O.P, 6, noncanon=False)
    out, ms = {}, {}
    for form in (0, 1):
        dx, dy = engine.to_device(x), engine.to_device(y)
        t = ctypes.c_float()
        assert probe.devapi_fp_rate(form, engine._ptr(dx), engine._ptr(dy), n, iters, ctypes.byref(t)) == 0
        torch.cuda.synchronize()
        out[form], ms[form] = engine.to_host(dx), t.value
    assert np.array_equal(out[0], out[1])
    # a few chains against the oracle: x y^(iters + 1) (the warm-up step included)
    for j in (5, 77, n - 1):
        exp = O.limbs_to_int(x[j]) * pow(O.limbs_to_int(y[j]), iters + 1, O.P) % O.P
        assert O.limbs_to_int(out[0][j]) == exp
    rate = {f: n * iters / (ms[f] * 1e-3) / 1e9 for f in ms}
    print(f"fp_mul device API: {rate[0]:.2f} G/s (2 products) vs {rate[1]:.2f} G/s (4 products)")
    assert ms[1] > 1.2 * ms[0]
