"""GPU parity of the Fr and G1 FFTs and the toeplitz gather against the oracle
and the reference's Fr FFT vector (fr_fft_testvector.cu), bit-exact."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu
R = O.R


def test_fr_fft_reference_vector(engine, kats):
    q = O.ints_to_array([int(h, 16) for h in kats["fr_fft"]["q"]], 4)
    a = [int(h, 16) % R for h in kats["fr_fft"]["a"]]
    dq = engine.to_device(q)
    out = engine.empty(q.shape)
    engine.call("fr_fft", engine._ptr(out), engine._ptr(dq), 1, engine._stream())
    assert [O.limbs_to_int(x) for x in engine.to_host(out)] == a
    # inverse, in place
    engine.call("fr_ift", engine._ptr(out), engine._ptr(out), 1, engine._stream())
    assert np.array_equal(engine.to_host(out), O.fr_op("reduce", q))


@pytest.mark.parametrize("log_m", [1, 2, 5, 7, 8, 9])
@pytest.mark.parametrize("inverse", [0, 1])
def test_fr_fft_sizes(engine, log_m, inverse):
    m = 1 << log_m
    x = O.seeded_fr(100 + log_m, 3 * m).reshape(3, m, 4)
    d = engine.to_device(x)
    out = engine.empty(x.shape)
    engine.call("fr_fft_n", engine._ptr(out), engine._ptr(d), log_m, 3, inverse, engine._stream())
    assert np.array_equal(engine.to_host(out), O.fr_fft(x, inverse=bool(inverse)))


def g1_points(seed, count):
    g = O.g1_generator().reshape(1, 18)
    ks = O.seeded_fr(seed, count)
    return O.g1_op("mul", np.repeat(g, count, 0), ks)


@pytest.mark.parametrize("log_m,count", [(3, 5), (6, 2), (9, 2)])
def test_g1_fft(engine, log_m, count):
    m = 1 << log_m
    pts = g1_points(log_m, count * m).reshape(count, m, 18)
    pts[0, 1] = 0
    pts[0, 1, 6] = 1  # an infinity among the inputs
    d = engine.to_device(pts)
    out = engine.empty(pts.shape)
    engine.call("g1p_fft_n", engine._ptr(out), engine._ptr(d), log_m, count, 0, engine._stream())
    fwd = O.g1_normalize(engine.to_host(out).reshape(-1, 18)).reshape(pts.shape)
    assert np.array_equal(fwd, O.g1_fft(pts))
    back = engine.empty(pts.shape)
    engine.call("g1p_fft_n", engine._ptr(back), engine._ptr(out), log_m, count, 1, engine._stream())
    assert np.array_equal(O.g1_normalize(engine.to_host(back).reshape(-1, 18)), O.g1_normalize(pts.reshape(-1, 18)))


def test_g1_ift_matches_oracle(engine):
    pts = g1_points(77, 2 * 512).reshape(2, 512, 18)
    d = engine.to_device(pts)
    out = engine.empty(pts.shape)
    engine.call("g1p_ift", engine._ptr(out), engine._ptr(d), 2, engine._stream())
    assert np.array_equal(O.g1_normalize(engine.to_host(out).reshape(-1, 18)).reshape(pts.shape),
                          O.g1_fft(pts, inverse=True))


def test_g1_fft_linearity_full_batch(engine):
    """FFT(a + b) == FFT(a) + FFT(b) over 40 rows of 512 (size-independent check)."""
    rows = 40
    a = g1_points(1, rows * 512)
    b = g1_points(2, rows * 512)
    da, db = engine.to_device(a), engine.to_device(b)
    dsum = engine.empty(a.shape)
    st = engine._stream()
    engine.call("g1p_op_n", engine.G1_OPS["add"], engine._ptr(dsum), engine._ptr(da), engine._ptr(db), len(a), st)
    fa, fb, fs = engine.empty(a.shape), engine.empty(a.shape), engine.empty(a.shape)
    engine.call("g1p_fft", engine._ptr(fa), engine._ptr(da), rows, st)
    engine.call("g1p_fft", engine._ptr(fb), engine._ptr(db), rows, st)
    engine.call("g1p_fft", engine._ptr(fs), engine._ptr(dsum), rows, st)
    fab = engine.empty(a.shape)
    engine.call("g1p_op_n", engine.G1_OPS["add"], engine._ptr(fab), engine._ptr(fa), engine._ptr(fb), len(a), st)
    import torch
    eq = torch.zeros(len(a), dtype=torch.uint8, device="cuda")
    import ctypes
    engine.call("g1p_eq_n", ctypes.c_void_p(eq.data_ptr()), engine._ptr(fab), engine._ptr(fs), len(a), st)
    assert int(eq.sum()) == len(a)


def test_toeplitz(engine):
    rows = 3
    poly = O.seeded_fr(55, rows * 4096).reshape(rows, 4096, 4)
    d = engine.to_device(poly)
    out = engine.empty((rows, 16, 512, 4))
    engine.call("fk20_poly2toeplitz_coefficients", engine._ptr(out), engine._ptr(d), rows, engine._stream())
    got = engine.to_host(out)
    for r in range(rows):
        assert np.array_equal(got[r], O.toeplitz(poly[r]))
    engine.call("fk20_poly2toeplitz_coefficients_fft", engine._ptr(out), engine._ptr(d), rows, engine._stream())
    got = engine.to_host(out)
    for r in range(rows):
        assert np.array_equal(got[r], O.fr_fft(O.toeplitz(poly[r])))
