"""The reference's false-positive defences and property tests, on the engine
(fk20_512test.cu:32-39 canaries, test.h:116-122 mangled expectations that must
fail, g1test_fft.cu:197-207 a planted point that must change the transform,
fptest/frtest algebraic properties, g1test_dbl.cu:18-56 p + p == dbl(p)), and
the FK20 test input of the reference's own harness: the Fibonacci polynomial
and fixed tau of FK20Py/fk20_multi_cuda.py:290-313."""
import ctypes

import numpy as np
import pytest

import oracle as O
from conftest import fk20_setup_data

pytestmark = pytest.mark.gpu

CANARY = 0xAAAAAAAAAAAAAAAA


def canaried(engine, shape):
    import torch
    t = engine.empty(shape)
    t.view(torch.int64).fill_(np.int64(np.uint64(CANARY).view(np.int64)))
    return t


def mangle(a: np.ndarray) -> np.ndarray:
    """A reversible one-bit change of a copy (varMangle, fk20_512test.cu:971-1008)."""
    b = a.copy()
    flat = b.reshape(-1)
    flat[len(flat) // 3] ^= np.uint64(1 << 17)
    return b


def test_canaried_pipeline_and_negative_check(engine):
    n, rows, m = 2048, 3, 256
    _, _, xext = fk20_setup_data(n)
    c = engine.Context(0, 8)
    c.load_xext_fft(n, engine.to_device(xext))
    poly = O.seeded_fr(8100, rows * n).reshape(rows, n, 4)
    dpoly = engine.to_device(poly)
    h = canaried(engine, (rows, m, 18))
    c.poly2h_fft(h, dpoly, rows, n)
    got = engine.to_host(h)
    assert not np.any(got == np.uint64(CANARY)), "an output element was not written"
    exp = O.fk20_rows(poly, xext)
    norm = O.g1_normalize(got.reshape(-1, 18)).reshape(got.shape)
    assert np.array_equal(norm, exp)
    assert not np.array_equal(norm, mangle(exp)), "the comparison must be able to fail"
    c.close()


def test_g1_fft_planted_point_changes_the_transform(engine):
    g = O.g1_generator().reshape(1, 18)
    pts = O.g1_op("mul", np.repeat(g, 512, 0), O.seeded_fr(8200, 512)).reshape(1, 512, 18)
    d = engine.to_device(pts)
    out = canaried(engine, (1, 512, 18))
    engine.call("g1p_fft_n", engine._ptr(out), engine._ptr(d), 9, 1, 0, engine._stream())
    exp = O.g1_fft(pts)
    got = O.g1_normalize(engine.to_host(out).reshape(-1, 18)).reshape(exp.shape)
    assert np.array_equal(got, exp)
    planted = pts.copy()
    planted[0, 511] = g[0]
    dp = engine.to_device(planted)
    engine.call("g1p_fft_n", engine._ptr(out), engine._ptr(dp), 9, 1, 0, engine._stream())
    got2 = O.g1_normalize(engine.to_host(out).reshape(-1, 18)).reshape(exp.shape)
    assert not np.array_equal(got2, exp)


@pytest.mark.parametrize("field", ["fp", "fr"])
def test_field_properties(engine, field):
    """a b = b a, (a + b) c = a c + b c, a (b c) = (a b) c, a a = sqr(a), a inv(a) = 1."""
    import torch
    limbs, mod, fn = (6, O.P, "fp_op_n") if field == "fp" else (4, O.R, "fr_op_n")
    rng = np.random.default_rng(31)
    cnt = 4096
    vals = [O.ints_to_array([int.from_bytes(rng.bytes(8 * limbs), "little") % mod for _ in range(cnt)], limbs)
            for _ in range(3)]
    a, b, c = (engine.to_device(v) for v in vals)
    ops = engine.FIELD_OPS

    def op(name, x, y=None):
        out = engine.empty(x.shape)
        engine.call(fn, ops[name], engine._ptr(out), engine._ptr(x), engine._ptr(y), cnt, engine._stream())
        return out

    assert torch.equal(op("mul", a, b), op("mul", b, a))
    assert torch.equal(op("mul", op("add", a, b), c), op("add", op("mul", a, c), op("mul", b, c)))
    assert torch.equal(op("mul", a, op("mul", b, c)), op("mul", op("mul", a, b), c))
    assert torch.equal(op("mul", a, a), op("sqr", a))
    one = op("mul", a, op("inv", a))
    assert np.array_equal(engine.to_host(one), O.ints_to_array([1] * cnt, limbs))


def test_g1_double_equals_self_add(engine):
    """p + p == dbl(p) for 20,000 points (g1test_dbl.cu:18-56)."""
    import torch
    g = O.g1_generator().reshape(1, 18)
    cnt = 20000
    base = engine.to_device(np.repeat(g, cnt, 0))
    scal = engine.to_device(O.seeded_fr(8300, cnt))
    p = engine.empty((cnt, 18))
    st = engine._stream()
    engine.call("g1p_op_n", engine.G1_OPS["mul"], engine._ptr(p), engine._ptr(base), engine._ptr(scal), cnt, st)
    s, d = engine.empty((cnt, 18)), engine.empty((cnt, 18))
    engine.call("g1p_op_n", engine.G1_OPS["add"], engine._ptr(s), engine._ptr(p), engine._ptr(p), cnt, st)
    engine.call("g1p_op_n", engine.G1_OPS["dbl"], engine._ptr(d), engine._ptr(p), None, cnt, st)
    eq = torch.zeros(cnt, dtype=torch.uint8, device="cuda")
    engine.call("g1p_eq_n", ctypes.c_void_p(eq.data_ptr()), engine._ptr(s), engine._ptr(d), cnt, st)
    assert int(eq.sum()) == cnt


def test_reference_harness_input(engine):
    """The reference's FK20 test case: the 4096-coefficient Fibonacci polynomial
    (x, y = 1, 1; pairs [x, y], x += y, y += x, mod r) against the setup of
    tau = 1927409816240961209460912649124 (FK20Py/fk20_multi_cuda.py:290-313)."""
    n, m = 4096, 512
    x, y, coeffs = 1, 1, []
    for _ in range(n // 2):
        x %= O.R
        y %= O.R
        coeffs += [x, y]
        x += y
        y += x
    poly = O.ints_to_array(coeffs, 4).reshape(1, n, 4)
    tau = O.int_to_limbs(1927409816240961209460912649124 % O.R, 4)
    setup = O.setup(tau, n + 1)
    xext = O.xext_fft(setup, n, 16)
    c = engine.Context(0, 8)
    c.load_setup(n, engine.to_device(setup))  # xext_fft computed on the GPU from the setup
    h = canaried(engine, (1, m, 18))
    c.poly2h_fft(h, engine.to_device(poly), 1, n)
    exp = O.fk20_row(poly[0], xext)["h_fft"]
    assert np.array_equal(O.g1_normalize(engine.to_host(h)[0]), exp)
    # and in the data-availability format
    import torch
    proofs = torch.zeros((1, m, 48), dtype=torch.uint8, device="cuda")
    c.poly2proofs(proofs, engine.to_device(poly), 1, n)
    assert np.array_equal(proofs.cpu().numpy(), O.da_proofs(exp.reshape(1, m, 18)))
    c.close()
