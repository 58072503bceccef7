"""Pairing checks on the GPU (kernels_pairing.cu), against the pure-Python
restatement oracle/pairing_py.py: G2 operations, pairing values bit-exact,
bilinearity, and the verification of FK20 proofs as KZG multiproofs
(check_proof_multi, FK20Py/kzg_proofs.py:207-232):
e(C - [r_j(s)]G1, G2) == e(proof_j, [s^16 - w^j]G2) with f = q_j (X^16 - w^j) + r_j."""
import numpy as np
import pytest

import oracle as O
import pairing_py as PP
from conftest import fk20_setup_data

pytestmark = pytest.mark.gpu


def g2_to_array(pts):
    """affine python G2 points (None = infinity) -> g2p_t rows (36 words)"""
    out = np.zeros((len(pts), 36), np.uint64)
    for i, q in enumerate(pts):
        if q is None:
            out[i, 12] = 1
            continue
        for k, v in enumerate((q[0][0], q[0][1], q[1][0], q[1][1], 1, 0)):
            out[i, 6 * k:6 * k + 6] = O.int_to_limbs(v, 6)
    return out


def g2_from_array(a):
    res = []
    for row in a:
        v = [O.limbs_to_int(row[6 * k:6 * k + 6]) for k in range(6)]
        res.append(None if v[4] == 0 and v[5] == 0 else ((v[0], v[1]), (v[2], v[3])))
    return res


def g1mul(k):
    g = O.g1_generator().reshape(1, 18)
    return O.g1_op("mul", g, O.int_to_limbs(k % O.R, 4).reshape(1, 4))[0]


def to_py(p18):
    return (O.limbs_to_int(p18[0:6]), O.limbs_to_int(p18[6:12]))


def test_g2_operations(engine):
    G2 = PP.g2_generator()
    ks = [5, 0xDEADBEEF, O.R - 1, O.R]
    a = engine.to_device(g2_to_array([G2] * len(ks)))
    s = engine.to_device(np.stack([O.int_to_limbs(k, 4) for k in ks]))
    out = engine.empty((len(ks), 36))
    engine.call("g2p_op_n", engine.G2_OPS["mul"], engine._ptr(out), engine._ptr(a), engine._ptr(s), len(ks),
                engine._stream())
    got = g2_from_array(engine.to_host(out))
    assert got == [PP.g2mul(k, G2) for k in ks]  # [r]G2 = infinity
    import torch
    flags = torch.zeros(len(ks), dtype=torch.uint8, device="cuda")
    engine.call("g2p_op_n", engine.G2_OPS["is_point"], None, engine._ptr(out), engine._ptr(flags), len(ks),
                engine._stream())
    assert flags.cpu().numpy().tolist() == [1, 1, 1, 1]


def test_pairing_values_match_restatement(engine):
    G2 = PP.g2_generator()
    a1, b1 = 3, 7
    p = np.stack([g1mul(1), g1mul(a1)])
    q = [G2, PP.g2mul(b1, G2)]
    out = engine.empty((2, 12, 6))
    dp, dq = engine.to_device(p), engine.to_device(g2_to_array(q))
    engine.call("fk20_pairing_n", engine._ptr(out), engine._ptr(dp), engine._ptr(dq), 2, engine._stream())
    got = engine.to_host(out)
    for i in range(2):
        exp = PP.pairing(to_py(p[i]), q[i])
        vals = [O.limbs_to_int(got[i, k]) for k in range(12)]
        assert vals == [c for pair in exp for c in pair], i


def test_pairing_checks_bilinear_and_negative(engine):
    G2 = PP.g2_generator()
    rng = np.random.default_rng(9)
    cases, expect = [], []
    for t in range(6):
        a = int.from_bytes(rng.bytes(31), "little")
        b = int.from_bytes(rng.bytes(31), "little")
        good = t % 2 == 0
        cases.append((g1mul(a), PP.g2mul(b, G2), g1mul(a * b + (0 if good else 1)), G2))
        expect.append(1 if good else 0)
    inf1 = np.zeros(18, np.uint64)
    inf1[6] = 1
    cases.append((inf1, G2, g1mul(5), None))  # e(O, Q) == e(P, O) == 1
    expect.append(1)
    A = engine.to_device(np.stack([c[0] for c in cases]))
    B = engine.to_device(g2_to_array([c[1] for c in cases]))
    C = engine.to_device(np.stack([c[2] for c in cases]))
    D = engine.to_device(g2_to_array([c[3] for c in cases]))
    import torch
    ok = torch.zeros(len(cases), dtype=torch.uint8, device="cuda")
    engine.call("fk20_pairing_check_n", engine._ptr(ok), engine._ptr(A), engine._ptr(B), engine._ptr(C),
                engine._ptr(D), len(cases), engine._stream())
    assert ok.cpu().numpy().tolist() == expect


def test_fk20_proofs_verify_as_kzg_multiproofs(engine):
    """Proofs and commitment from the engine, checked with pairings; a proof
    paired with the wrong coset must fail."""
    import torch
    n, m = 4096, 512
    tau, setup, xext = fk20_setup_data(n)
    t = O.limbs_to_int(tau)
    poly = O.seeded_fr(9100, n).reshape(1, n, 4)
    c = engine.Context(0, 8)
    c.load_xext_fft(n, engine.to_device(xext))
    c.load_commit(n, engine.to_device(setup[:n]), 8)
    dpoly = engine.to_device(poly)
    h = engine.empty((1, m, 18))
    c.poly2h_fft(h, dpoly, 1, n)
    com = engine.empty((1, 18))
    c.commit(com, dpoly, 1, n)
    f = [O.limbs_to_int(x) for x in poly[0]]
    w = O.root_of_unity(512)
    js = [0, 1, 255, 511]
    rem = np.zeros((len(js), 32, 4), np.uint64)  # r_j = f mod (X^16 - w^j), padded to 32 coefficients
    s2 = []
    for i, j in enumerate(js):
        cj = pow(w, j, O.R)
        for k in range(16):
            v = sum(f[k + 16 * q] * pow(cj, q, O.R) for q in range(n // 16)) % O.R
            rem[i, k] = O.int_to_limbs(v, 4)
        s2.append((pow(t, 16, O.R) - cj) % O.R)
    R = engine.empty((len(js), 18))
    c.commit(R, engine.to_device(rem), len(js), 32)
    lhs = engine.empty((len(js), 18))
    comr = engine.to_device(np.repeat(engine.to_host(com), len(js), axis=0))
    engine.call("g1p_op_n", engine.G1_OPS["sub"], engine._ptr(lhs), engine._ptr(comr), engine._ptr(R), len(js),
                engine._stream())
    G2 = PP.g2_generator()
    g2s = engine.to_device(g2_to_array([G2] * (2 * len(js))))
    scal = engine.to_device(np.stack([O.int_to_limbs(v, 4) for v in s2 + s2]))
    rhs2 = engine.empty((2 * len(js), 36))
    engine.call("g2p_op_n", engine.G2_OPS["mul"], engine._ptr(rhs2), engine._ptr(g2s), engine._ptr(scal),
                2 * len(js), engine._stream())
    hh = engine.to_host(h)[0]
    proofs = engine.to_device(np.concatenate([hh[js], hh[[(j + 1) % m for j in js]]]))  # right coset, then a wrong one
    A = engine.to_device(np.concatenate([engine.to_host(lhs)] * 2))
    B = engine.to_device(g2_to_array([G2] * (2 * len(js))))
    ok = torch.zeros(2 * len(js), dtype=torch.uint8, device="cuda")
    engine.call("fk20_pairing_check_n", engine._ptr(ok), engine._ptr(A), engine._ptr(B), engine._ptr(proofs),
                engine._ptr(rhs2), 2 * len(js), engine._stream())
    assert ok.cpu().numpy().tolist() == [1] * len(js) + [0] * len(js)
    c.close()
