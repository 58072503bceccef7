"""The CPU oracle pinned against the reference's own known answers.

Golden vectors come from the reference's KAT kernels (tests/golden/reference_kats.json,
made by tests/golden/make_reference_kats.py from fptest_kat.cu, frtest_kat.cu,
g1test_kat.cu, fr_fft_testvector.cu, fr_roots.cu).  The reference compares through
fp_neq / fr_neq / g1p_neq, i.e. modulo p / r and after projective normalisation,
so the same relation is used here.  The FK20 pipeline itself is pinned by the
pairing-free KZG identity and by the pure-Python restatement of FK20Py.
"""
import numpy as np
import pytest

import oracle as O
from conftest import kzg_multi_case
import fk20_py as PY

P, R = O.P, O.R


def h2i(h):
    return int(h, 16)


def arr(hexes, n):
    return O.ints_to_array([h2i(h) for h in hexes], n)


def ints(a):
    return [O.limbs_to_int(r) for r in np.asarray(a)]


@pytest.mark.parametrize("field", ["fp", "fr"])
def test_field_kats(kats, field):
    n, mod, op_fn = (6, P, O.fp_op) if field == "fp" else (4, R, O.fr_op)
    checked = 0
    for k in kats[field]:
        op = k["op"]
        if op == "cpy":
            continue
        if op == "reduce":
            got = ints(op_fn("reduce", arr(k["q"], n)))
            assert got == [h2i(a) for a in k["a"]], "reduce"
            checked += len(got)
        elif op == "eq":
            t = [h2i(x) % mod for x in k["t"]]
            u = [h2i(x) % mod for x in k["u"]]
            for i in range(len(t)):
                for j in range(len(u)):
                    assert (t[i] == u[j]) == (i == j)
            checked += 1
        elif op in ("neg", "x2", "x3", "sqr", "inv"):
            got = ints(op_fn(op, arr(k["q"], n)))
            for g, a in zip(got, k["a"]):
                if k.get("exact"):
                    assert g == h2i(a), op
                else:
                    assert g == h2i(a) % mod, op
            checked += len(got)
        elif op in ("add", "sub", "mul"):
            got = ints(op_fn(op, arr(k["x"], n), arr(k["y"], n)))
            assert got == [h2i(a) % mod for a in k["a"]], op
            checked += len(got)
        elif op == "mandelbrot":
            for q, a in zip(k["q"], k["a"]):
                x = arr([q], n)
                z = np.zeros((1, n), np.uint64)
                for _ in range(k["iterations"]):
                    z = op_fn("add", op_fn("sqr", z), x)
                assert O.limbs_to_int(z[0]) == h2i(a) % mod
                checked += 1
        else:
            raise AssertionError(op)
    assert checked > 50


def g1p_from_kat(rows):
    return np.concatenate([O.int_to_limbs(h2i(r), 6) for r in rows]).reshape(1, 18)


def test_g1_kats(kats):
    g = O.g1_generator().reshape(1, 18)
    pts = {k: g1p_from_kat(v) for k, v in kats["g1"].items() if len(v) == 3}
    norm = {k: O.g1_normalize(v) for k, v in pts.items()}
    assert all(O.g1_is_point(v) for v in pts.values())
    two = O.g1_op("dbl", g)
    assert np.array_equal(two, norm["g1p_x2"])
    assert np.array_equal(O.g1_op("add", g, g), norm["g1p_x2"])
    three = O.g1_op("add", g, pts["g1p_x2"])
    assert np.array_equal(three, norm["g1p_x3"])
    t24 = O.g1_op("dbl", O.g1_op("dbl", O.g1_op("dbl", three)))
    assert np.array_equal(t24, norm["g1p_x24"])
    t25 = O.g1_op("add", O.g1_op("sub", t24, pts["g1p_x2"]), pts["g1p_x3"])
    assert np.array_equal(t25, norm["g1p_x25"])
    assert np.array_equal(O.g1_op("mul", g, O.int_to_limbs(25, 4).reshape(1, 4)), norm["g1p_x25"])
    # w^1 * G and w^8 * G with w = fr_roots[1] (g1test_kat.cu:262-285)
    w1 = h2i(kats["fr_roots"][1])
    wG = O.g1_op("mul", g, O.int_to_limbs(w1, 4).reshape(1, 4))
    assert np.array_equal(wG, norm["g1p_wG"])
    w8 = h2i(kats["fr_roots"][8])
    assert np.array_equal(O.g1_op("mul", g, O.int_to_limbs(w8, 4).reshape(1, 4)), norm["g1p_w8G"])
    # infinity: any (0, y != 0, 0) is the neutral element (g1test_kat.cu:11-18)
    inf = np.zeros((1, 18), np.uint64)
    inf[0, 6:12] = [1, 2, 3, 4, 5, 6]
    assert np.array_equal(O.g1_op("add", g, inf), O.g1_normalize(g))
    assert O.limbs_to_int(O.g1_normalize(inf)[0]) == 1 << (64 * 6)


def test_fr_roots_table(kats):
    roots = [h2i(x) for x in kats["fr_roots"]]
    w = O.root_of_unity(512)
    assert w == PY.get_root_of_unity(512)
    for i in range(513):
        assert roots[i] % R == pow(w, i, R)
    inv512 = pow(512, R - 2, R)
    assert roots[513] % R == inv512
    assert roots[514] % R == inv512 * pow(w, R - 1 - 128, R) % R


def test_fr_fft_vector(kats):
    q = arr(kats["fr_fft"]["q"], 4).reshape(512, 4)
    a = [h2i(x) % R for x in kats["fr_fft"]["a"]]
    got = ints(O.fr_fft(q))
    assert got == a
    back = O.fr_fft(O.fr_fft(q), inverse=True)
    assert np.array_equal(back, O.fr_op("reduce", q).reshape(512, 4))


def test_seeded_stream_matches_c():
    assert np.array_equal(O.seeded_fr(123, 5000), O.seeded_fr_c(123, 5000))
    v = O.seeded_fr(9, 2000)
    assert all(O.limbs_to_int(x) < R for x in v)


def _to_py_point(p18):
    z = O.limbs_to_int(p18[12:18])
    if z == 0:
        return None
    assert z == 1
    return (O.limbs_to_int(p18[0:6]), O.limbs_to_int(p18[6:12]))


@pytest.mark.parametrize("n", [64, 128])
def test_oracle_matches_python_restatement(n):
    l = 16
    tau = O.seeded_fr(77, 1)[0]
    poly = O.seeded_fr(78, n)
    setup = O.setup(tau, n + 1)
    xext = O.xext_fft(setup, n, l)
    res = O.fk20_row(poly, xext, l)
    py = PY.fk20_da([O.limbs_to_int(x) for x in poly], l, [_to_py_point(s) for s in setup])
    assert [[_to_py_point(p) for p in row] for row in xext] == py["xext_fft"]
    assert [ints(r) for r in res["tc"]] == py["tc"]
    assert [ints(r) for r in res["tc_fft"]] == py["tc_fft"]
    assert [_to_py_point(p) for p in res["hext_fft"]] == py["hext_fft"]
    assert [_to_py_point(p) for p in res["h"]] == py["h"]
    assert [_to_py_point(p) for p in res["h_fft"]] == py["h_fft"]


@pytest.mark.parametrize("n", [64, 256, 1024])
def test_oracle_kzg_identity(n):
    """h_fft[j] == [q_j(tau)] G1 with q_j = f div (X^16 - w_2k^j)."""
    tau = O.seeded_fr(5, 1)[0]
    poly = O.seeded_fr(6, n)
    xext = O.xext_fft(O.setup(tau, n + 1), n)
    res = O.fk20_row(poly, xext)
    m = 2 * n // 16
    js = list(range(0, m, max(1, m // 16)))
    direct = np.concatenate([O.kzg_direct(poly, tau, 16, j, j + 1) for j in js])
    assert np.array_equal(res["h_fft"][js], direct)


def test_toeplitz_matches_reference_kernel_indexing():
    """tc[i][(t+257)%512] = poly[16t+15-i] for t>0, tc[i][1..257]=0
    (fk20_poly2toeplitz_coefficients.cu:40-56)."""
    n = 4096
    poly = O.seeded_fr(11, n)
    tc = O.toeplitz(poly)
    exp = np.zeros((16, 512, 4), np.uint64)
    for i in range(16):
        for t in range(1, 256):
            exp[i, (t + 257) % 512] = poly[16 * t + 15 - i]
    assert np.array_equal(tc, exp)


def test_fk20_degenerate_inputs():
    """Zero polynomial -> every proof is infinity; linearity in the polynomial."""
    n, l = 128, 16
    tau = O.seeded_fr(3, 1)[0]
    xext = O.xext_fft(O.setup(tau, n + 1), n, l)
    zero = np.zeros((n, 4), np.uint64)
    res = O.fk20_row(zero, xext, l)
    inf = np.zeros(18, np.uint64)
    inf[6] = 1
    assert all(np.array_equal(p, inf) for p in res["h_fft"])
    a = O.seeded_fr(1, n)
    b = O.seeded_fr(2, n)
    s = O.fr_op("add", a, b)
    ha = O.fk20_row(a, xext, l)["h_fft"]
    hb = O.fk20_row(b, xext, l)["h_fft"]
    hs = O.fk20_row(s, xext, l)["h_fft"]
    assert np.array_equal(O.g1_op("add", ha, hb), hs)


def test_compressed_encoding_pins():
    """The published 48-byte encoding of the BLS12-381 G1 generator (x with the
    compression flag; its y is the smaller root), of its negation (sign flag
    set) and of the point at infinity."""
    g = O.g1_generator().reshape(1, 18)
    gen = "97f1d3a73197d7942695638c4fa9ac0fc3688c4f9774b905a14e3a3f171bac586c55e83ff97a1aeffb3af00adb22c6bb"
    assert O.g1_compress(g)[0].tobytes().hex() == gen
    neg = O.g1_compress(O.g1_op("neg", g))[0].tobytes().hex()
    assert neg == "b" + gen[1:]
    inf = np.zeros((1, 18), np.uint64)
    inf[0, 6] = 1
    assert O.g1_compress(inf)[0].tobytes() == bytes([0xC0]) + bytes(47)


def test_reverse_bit_order_matches_reference_definition():
    """list_to_reverse_bit_order (kzg_proofs.py:105-118) reverses the
    log2(m)-bit binary string of the index; applying it twice is the identity."""
    m = 16
    rows = np.arange(2 * m * 3).reshape(2, m, 3)
    r = O.reverse_bit_order(rows)
    for i in range(m):
        j = int(('{:0' + str(m.bit_length() - 1) + 'b}').format(i)[::-1], 2)
        assert np.array_equal(r[:, i], rows[:, j])
    assert np.array_equal(O.reverse_bit_order(r), rows)


def test_pairing_restatement_is_bilinear():
    """The pairing checker (oracle/pairing_py.py): non-degenerate, bilinear,
    and the verification equation holds exactly for matching exponents."""
    import pairing_py as PP
    g = O.g1_generator()

    def g1mul(k):
        p = O.g1_op("mul", g.reshape(1, 18), O.int_to_limbs(k % O.R, 4).reshape(1, 4))[0]
        return (O.limbs_to_int(p[0:6]), O.limbs_to_int(p[6:12]))

    G1, G2 = g1mul(1), PP.g2_generator()
    assert PP.g2mul(O.R, G2) is None  # the generator has order r
    e = PP.pairing(G1, G2)
    assert e != PP.ONE12 and PP.f12pow(e, O.R) == PP.ONE12
    a, b = 0x1234567890ABCDEF, 0xFEDCBA0987654321
    assert PP.pairing(g1mul(a), PP.g2mul(b, G2)) == PP.f12pow(e, a * b % O.R)
    assert PP.pairing_check(g1mul(a), PP.g2mul(b, G2), g1mul(a * b), G2)
    assert not PP.pairing_check(g1mul(a), PP.g2mul(b, G2), g1mul(a * b + 1), G2)


def test_check_proof_multi_restatement():
    """oracle/pairing_py.check_proof_multi (FK20Py/kzg_proofs.py:207-232)
    accepts a proof built from the KZG definitions and rejects a wrong value."""
    import pairing_py as PP
    c = kzg_multi_case()
    args = (c["setup_g1"], c["setup_g2"])
    assert PP.check_proof_multi(c["commitment"], c["proof"], c["x"], c["ys"], *args)
    bad = list(c["ys"])
    bad[1] = (bad[1] + 1) % O.R
    assert not PP.check_proof_multi(c["commitment"], c["proof"], c["x"], bad, *args)
