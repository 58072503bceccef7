"""The engine's field, curve and fixed-scalar-program code compiled for the
host (carry flag emulated, tests/host/emul.cpp) checked against the oracle.

This exercises the exact limb schedules, reduction bounds (including
non-canonical inputs up to 2^384 - 1), complete addition laws and GLV/NAF
programs that the kernels run, without a GPU.  It is test infrastructure:
the product library never runs this host build on its data path."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT

HOST = os.path.join(ROOT, "tests", "host")


@pytest.fixture(scope="module")
def emul(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("emul") / "libemul.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I",
                    os.path.join(ROOT, "fk20-cuda_b200", "csrc"), os.path.join(HOST, "emul.cpp"), "-o", so],
                   check=True)
    return ctypes.CDLL(so)


def P(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


def field_inputs(rng, count, mod, limbs):
    xs = [int.from_bytes(rng.bytes(8 * limbs), "little") % mod for _ in range(count)]
    edge = [0, 1, 2, mod - 1, mod - 2, mod // 2, (1 << (64 * limbs)) - 1, (1 << (64 * limbs)) - mod]
    xs[: len(edge)] = edge
    for j in range(8, 24):  # non-canonical representatives
        if xs[j] + mod < (1 << (64 * limbs)):
            xs[j] += mod
    return O.ints_to_array(xs, limbs)


@pytest.mark.parametrize("field", ["fp", "fr"])
def test_field_code_matches_oracle(emul, field):
    rng = np.random.default_rng(2)
    limbs, mod = (6, O.P) if field == "fp" else (4, O.R)
    fn = emul.emul_fp_op if field == "fp" else emul.emul_fr_op
    ofn = O.fp_op if field == "fp" else O.fr_op
    a = field_inputs(rng, 1500, mod, limbs)
    b = field_inputs(rng, 1500, mod, limbs)[::-1].copy()
    for op, code in (("mul", 0), ("sqr", 1), ("add", 2), ("sub", 3), ("neg", 4), ("inv", 5), ("reduce", 6),
                     ("x2", 7), ("x12", 11)):
        n = 100 if op == "inv" else len(a)
        two = op in ("mul", "add", "sub")
        out = np.zeros_like(a)
        assert fn(code, P(out), P(a), P(b) if two else None, n) == 0
        assert np.array_equal(out[:n], ofn(op, a[:n], b[:n] if two else None)), (field, op)


def test_curve_formulas_match_oracle(emul):
    rng = np.random.default_rng(3)
    g = O.g1_generator().reshape(1, 18)
    ks = [int.from_bytes(rng.bytes(32), "little") % O.R for _ in range(30)]
    pts = np.concatenate([O.g1_op("mul", g, O.int_to_limbs(k, 4).reshape(1, 4)) for k in ks])
    qts = np.concatenate([pts[3:], pts[:3]])
    inf = np.zeros((1, 18), np.uint64)
    inf[0, 6] = 1
    pts = np.concatenate([pts, inf, inf, g, g])
    qts = np.concatenate([qts, g, inf, g, O.g1_op("neg", g)])  # P+inf, inf+inf, P+P, P-P
    out = np.zeros_like(pts)
    emul.emul_g1_op(0, P(out), P(pts), P(qts), len(pts))
    assert np.array_equal(O.g1_normalize(out), O.g1_op("add", pts, qts))
    emul.emul_g1_op(1, P(out), P(pts), None, len(pts))
    assert np.array_equal(O.g1_normalize(out), O.g1_op("dbl", pts))
    aff = np.ascontiguousarray(O.g1_normalize(qts)[:, :12])
    finite = [i for i in range(len(qts)) if O.limbs_to_int(O.g1_normalize(qts)[i, 12:]) == 1]
    emul.emul_g1_op(2, P(out), P(pts), P(aff), len(pts))
    assert np.array_equal(O.g1_normalize(out)[finite], O.g1_op("add", pts, qts)[finite])
    lam = 0xAC45A4010001A40200000000FFFFFFFF
    emul.emul_g1_op(3, P(out), P(pts), None, len(pts))
    assert np.array_equal(O.g1_normalize(out), O.g1_op("mul", pts, np.tile(O.int_to_limbs(lam, 4), (len(pts), 1))))


def test_glv_programs_match_scalar_multiplication(emul):
    rng = np.random.default_rng(4)
    g = O.g1_generator().reshape(1, 18)
    ks = [int.from_bytes(rng.bytes(32), "little") % O.R for _ in range(3)]
    pts = np.concatenate([O.g1_op("mul", g, O.int_to_limbs(k, 4).reshape(1, 4)) for k in ks])
    inf = np.zeros((1, 18), np.uint64)
    inf[0, 6] = 1
    pts = np.concatenate([pts, inf])
    w = O.root_of_unity(512)
    scalars = [pow(w, t, O.R) for t in (1, 2, 100, 128, 255, 256, 257, 384, 511)]
    scalars += [0, 1, O.R - 1, pow(512, O.R - 2, O.R), pow(2, O.R - 2, O.R)]
    for k in scalars:
        out = np.zeros_like(pts)
        d, a = ctypes.c_int(), ctypes.c_int()
        emul.emul_g1_mul_prog(P(out), P(pts), P(O.int_to_limbs(k, 4)), len(pts), ctypes.byref(d), ctypes.byref(a))
        exp = O.g1_op("mul", pts, np.tile(O.int_to_limbs(k, 4), (len(pts), 1)))
        assert np.array_equal(O.g1_normalize(out), exp), hex(k)
        assert d.value <= 129 and a.value <= 100
