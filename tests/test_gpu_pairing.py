"""Pairing checks on the GPU (kernels_pairing.cu), against the pure-Python
restatement oracle/pairing_py.py: G2 operations, pairing values bit-exact,
bilinearity, and the verification of FK20 proofs as KZG multiproofs
(check_proof_multi, FK20Py/kzg_proofs.py:207-232):
e(C - [r_j(s)]G1, G2) == e(proof_j, [s^16 - w^j]G2) with f = q_j (X^16 - w^j) + r_j."""
import numpy as np
import pytest

import oracle as O
import pairing_py as PP
from conftest import fk20_setup_data, kzg_multi_case

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


def g1_to_array(pts):
    """affine python G1 points -> g1p_t rows (z = 1)"""
    out = np.zeros((len(pts), 18), np.uint64)
    for i, q in enumerate(pts):
        out[i, 0:6] = O.int_to_limbs(q[0], 6)
        out[i, 6:12] = O.int_to_limbs(q[1], 6)
        out[i, 12] = 1
    return out


def test_check_proof_multi_on_engine_proofs(engine):
    """fk20_ctx_check_proof_multi (check_proof_multi, FK20Py/kzg_proofs.py:207-232)
    on the engine's own proofs: h_fft[j] proves the coset x w16^k with
    x = w8192^j (the data-availability checks of fk20_multi.py:154-165 use
    x = w8192^rbo(pos) for proof pos of the bit-reversed list).  Valid proofs
    pass; a wrong value, a proof of another coset and another polynomial's
    commitment fail.  A second call with l = 4 checks a proof built from the
    KZG definitions, against the restatement's verdicts."""
    import torch
    n, m, l = 4096, 512, 16
    tau, setup, xext = fk20_setup_data(n)
    t = O.limbs_to_int(tau)
    polys = O.seeded_fr(9200, 2 * n).reshape(2, n, 4)
    c = engine.Context(0, 8)
    c.load_xext_fft(n, engine.to_device(xext))
    c.load_commit(n, engine.to_device(setup[:n]), 8)
    dpolys = engine.to_device(polys)
    h = engine.empty((1, m, 18))
    c.poly2h_fft(h, dpolys[0:1], 1, n)
    com = engine.empty((2, 18))
    c.commit(com, dpolys, 2, n)
    hh, cc = engine.to_host(h)[0], engine.to_host(com)
    f = [O.limbs_to_int(v) for v in polys[0]]

    def evalf(z):
        acc = 0
        for coef in reversed(f):
            acc = (acc * z + coef) % O.R
        return acc

    w8192, w16 = O.root_of_unity(2 * n), O.root_of_unity(16)
    js = [0, 1, 77, 255, 256, 511]
    xs = [pow(w8192, j, O.R) for j in js]
    yss = [[evalf(x * pow(w16, k, O.R) % O.R) for k in range(l)] for x in xs]
    bad_ys = list(yss[0])
    bad_ys[3] = (bad_ys[3] + 1) % O.R
    cases = [(cc[0], hh[j], x, ys) for j, x, ys in zip(js, xs, yss)]
    cases += [(cc[0], hh[js[0]], xs[0], bad_ys),  # a wrong value
              (cc[0], hh[js[1] + 1], xs[1], yss[1]),  # the proof of another coset
              (cc[1], hh[js[2]], xs[2], yss[2])]  # another polynomial's commitment
    expect = [1] * len(js) + [0, 0, 0]
    G2 = PP.g2_generator()
    setup_g2 = engine.to_device(g2_to_array([PP.g2mul(pow(t, k, O.R), G2) for k in range(l + 1)]))
    dev = lambda a: engine.to_device(np.ascontiguousarray(a))
    C = dev(np.stack([q[0] for q in cases]))
    Pf = dev(np.stack([q[1] for q in cases]))
    X = dev(np.stack([O.int_to_limbs(q[2], 4) for q in cases]))
    Y = dev(np.stack([np.stack([O.int_to_limbs(v, 4) for v in q[3]]) for q in cases]))
    ok = torch.zeros(len(cases), dtype=torch.uint8, device="cuda")
    c.check_proof_multi(ok, C, Pf, X, Y, l, setup_g2, len(cases))
    assert ok.cpu().numpy().tolist() == expect

    # l = 4, a proof from the definitions (same tau as the context's tables)
    small = kzg_multi_case(l=4, tau=t)
    bad = list(small["ys"])
    bad[1] = (bad[1] + 1) % O.R
    verdicts = [PP.check_proof_multi(small["commitment"], small["proof"], small["x"], ys, small["setup_g1"],
                                     small["setup_g2"]) for ys in (small["ys"], bad)]
    assert verdicts == [True, False]
    C4 = dev(g1_to_array([small["commitment"]] * 2))
    P4 = dev(g1_to_array([small["proof"]] * 2))
    X4 = dev(np.stack([O.int_to_limbs(small["x"], 4)] * 2))
    Y4 = dev(np.stack([np.stack([O.int_to_limbs(v, 4) for v in ys]) for ys in (small["ys"], bad)]))
    ok4 = torch.zeros(2, dtype=torch.uint8, device="cuda")
    c.check_proof_multi(ok4, C4, P4, X4, Y4, 4, dev(g2_to_array(small["setup_g2"])), 2)
    assert [bool(v) for v in ok4.cpu().numpy()] == verdicts
    c.close()
