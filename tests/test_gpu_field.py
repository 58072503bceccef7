"""GPU parity of the field and curve layer (fp_op_n, fr_op_n, g1p_op_n, eq and
affine helpers) against the oracle and the reference's KAT vectors
(fptest_kat.cu, frtest_kat.cu, g1test_kat.cu).  Bit-exact: outputs are
canonical field elements; points are compared after affine normalisation."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

P, R = O.P, O.R


def rand_field(rng, count, mod, limbs):
    xs = [int.from_bytes(rng.bytes(8 * limbs), "little") % mod for _ in range(count)]
    edge = [0, 1, 2, mod - 1, mod - 2, mod // 2, mod // 2 + 1, (1 << (64 * limbs - 1)) % mod]
    xs[: len(edge)] = edge
    # weakly reduced representatives (any value < 2^(64*limbs)) as the reference allows
    for j in range(8, 16):
        xs[j] = xs[j] + mod if xs[j] + mod < (1 << (64 * limbs)) else xs[j]
    xs[16] = (1 << (64 * limbs)) - 1
    return O.ints_to_array(xs, limbs)


@pytest.mark.parametrize("field", ["fp", "fr"])
def test_field_ops_random(engine, field):
    rng = np.random.default_rng(11)
    limbs, mod = (6, P) if field == "fp" else (4, R)
    a = rand_field(rng, 3000, mod, limbs)
    b = rand_field(rng, 3000, mod, limbs)[::-1].copy()
    da, db = engine.to_device(a), engine.to_device(b)
    out = engine.empty(a.shape)
    oracle_op = O.fp_op if field == "fp" else O.fr_op
    fn = "fp_op_n" if field == "fp" else "fr_op_n"
    for op in ("mul", "sqr", "add", "sub", "neg", "x2", "x3", "x4", "x8", "x12", "reduce", "inv"):
        n = 300 if op == "inv" else len(a)
        two = op in ("mul", "add", "sub")
        engine.call(fn, engine.FIELD_OPS[op], engine._ptr(out), engine._ptr(da), engine._ptr(db) if two else None, n,
                    engine._stream())
        got = engine.to_host(out)[:n]
        exp = oracle_op(op, a[:n], b[:n] if two else None)
        assert np.array_equal(got, exp), (field, op)


@pytest.mark.parametrize("field", ["fp", "fr"])
def test_field_kats(engine, kats, field):
    limbs, mod = (6, P) if field == "fp" else (4, R)
    fn = "fp_op_n" if field == "fp" else "fr_op_n"

    def run(op, x, y=None):
        dx = engine.to_device(O.ints_to_array([int(h, 16) for h in x], limbs))
        dy = engine.to_device(O.ints_to_array([int(h, 16) for h in y], limbs)) if y else None
        out = engine.empty(dx.shape)
        engine.call(fn, engine.FIELD_OPS[op], engine._ptr(out), engine._ptr(dx), engine._ptr(dy), len(x),
                    engine._stream())
        return [O.limbs_to_int(r) for r in engine.to_host(out)]

    for k in kats[field]:
        op = k["op"]
        if op == "reduce":
            assert run("reduce", k["q"]) == [int(a, 16) for a in k["a"]]
        elif op in ("neg", "x2", "x3", "sqr", "inv"):
            assert run(op, k["q"]) == [int(a, 16) % mod for a in k["a"]], op
        elif op in ("add", "sub", "mul"):
            assert run(op, k["x"], k["y"]) == [int(a, 16) % mod for a in k["a"]], op


def test_g1_ops(engine, kats):
    rng = np.random.default_rng(5)
    g = O.g1_generator().reshape(1, 18)
    ks = [int.from_bytes(rng.bytes(32), "little") % R for _ in range(40)]
    pts = np.concatenate([O.g1_op("mul", g, O.int_to_limbs(k, 4).reshape(1, 4)) for k in ks])
    qts = np.concatenate([pts[1:], pts[:1]])
    inf = np.zeros((1, 18), np.uint64)
    inf[0, 6:12] = [1, 2, 3, 4, 5, 6]  # any (0, y != 0, 0), g1test_kat.cu:11-18
    x2 = np.concatenate([O.int_to_limbs(int(h, 16), 6) for h in kats["g1"]["g1p_x2"]]).reshape(1, 18)
    pts = np.concatenate([pts, inf, g, g, x2, g])
    qts = np.concatenate([qts, g, g, O.g1_op("neg", g), inf, x2])
    dp, dq = engine.to_device(pts), engine.to_device(qts)
    out = engine.empty(pts.shape)
    st = engine._stream()
    for op in ("add", "sub", "dbl", "neg", "normalize"):
        two = op in ("add", "sub")
        engine.call("g1p_op_n", engine.G1_OPS[op], engine._ptr(out), engine._ptr(dp), engine._ptr(dq) if two else None,
                    len(pts), st)
        got = O.g1_normalize(engine.to_host(out))
        exp = O.g1_op(op if op != "normalize" else "normalize", pts, qts if two else None)
        assert np.array_equal(got, exp), op
    scal = np.stack([O.int_to_limbs(int.from_bytes(rng.bytes(32), "little"), 4) for _ in range(len(pts))])
    dscal = engine.to_device(scal)
    engine.call("g1p_op_n", engine.G1_OPS["mul"], engine._ptr(out), engine._ptr(dp), engine._ptr(dscal), len(pts), st)
    assert np.array_equal(O.g1_normalize(engine.to_host(out)), O.g1_op("mul", pts, scal))
    # is_point on valid points, a broken point and the ANYINF infinity
    bad = pts.copy()
    bad[3, 0] ^= np.uint64(1)
    import torch
    flags = torch.zeros(len(pts), dtype=torch.uint8, device="cuda")
    dbad = engine.to_device(bad)
    engine.call("g1p_op_n", engine.G1_OPS["is_point"], None, engine._ptr(dbad), ctypes_ptr(flags), len(pts), st)
    f = flags.cpu().numpy()
    assert f[3] == 0 and f.sum() == len(pts) - 1


def ctypes_ptr(t):
    import ctypes
    return ctypes.c_void_p(t.data_ptr())


def test_eq_and_affine(engine):
    import torch
    g = O.g1_generator().reshape(1, 18)
    rng = np.random.default_rng(9)
    ks = [int.from_bytes(rng.bytes(32), "little") % R for _ in range(16)]
    pts = np.concatenate([O.g1_op("mul", g, O.int_to_limbs(k, 4).reshape(1, 4)) for k in ks])
    # a projective rescaling of the same points: (X z, Y z, z) for z = 7
    sc = pts.copy()
    for r in range(len(sc)):
        for c in range(2):
            v = O.limbs_to_int(sc[r, 6 * c:6 * c + 6]) * 7 % P
            sc[r, 6 * c:6 * c + 6] = O.int_to_limbs(v, 6)
        sc[r, 12:18] = O.int_to_limbs(7, 6)
    sc[5] = pts[6]
    eq = torch.zeros(len(pts), dtype=torch.uint8, device="cuda")
    # keep every device buffer referenced until the kernels that read it are enqueued
    dpts, dsc = engine.to_device(pts), engine.to_device(sc)
    engine.call("g1p_eq_n", ctypes_ptr(eq), engine._ptr(dpts), engine._ptr(dsc), len(pts), engine._stream())
    e = eq.cpu().numpy()
    assert e[5] == 0 and e.sum() == len(pts) - 1
    aff = engine.empty((len(pts), 12))
    engine.call("g1a_fromG1p_n", engine._ptr(aff), engine._ptr(dsc), len(pts), engine._stream())
    assert np.array_equal(engine.to_host(aff), O.g1_normalize(sc)[:, :12])
    a = O.ints_to_array([1, 2, R + 1, R - 1], 4)
    b = O.ints_to_array([1, 3, 1, 2 * R - 1], 4)
    eqr = torch.zeros(4, dtype=torch.uint8, device="cuda")
    da, db = engine.to_device(a), engine.to_device(b)
    engine.call("fr_eq_n", ctypes_ptr(eqr), engine._ptr(da), engine._ptr(db), 4, engine._stream())
    assert eqr.cpu().numpy().tolist() == [1, 0, 1, 1]
