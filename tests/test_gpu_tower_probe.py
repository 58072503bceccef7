"""The pairing's sparse line product (fk20-cuda_b200/csrc/tower.cuh,
f12_mul_line) against the restatement's Fp12 product (oracle/pairing_py.py),
in the library's code arrangement and in the arrangement with the Fp6 sums as
rolled loops (tests/host/tower_probe.cu).

The rolled arrangement once gave wrong values on the GPU.  Making every carry
chain one asm statement did not change that (the probe, built against the
field code with separate one-instruction statements and against the new one,
failed the same way); what did is passing values instead of pointers to the
out-of-line Fp2 products.  Both arrangements must now equal the restatement
on every element."""
import ctypes
import os
import random
import subprocess

import numpy as np
import pytest

import pairing_py as PP
from conftest import ROOT

pytestmark = pytest.mark.gpu
HOST = os.path.join(ROOT, "tests", "host")
RM = 1 << 384


def words(x):  # Montgomery form, 12 little-endian 32-bit words
    m = x * RM % PP.P
    return [(m >> (32 * k)) & 0xFFFFFFFF for k in range(12)]


def unwords(ws):
    m = sum(int(w) << (32 * k) for k, w in enumerate(ws))
    return m * pow(RM, -1, PP.P) % PP.P


STRUCT_ORDER = (0, 2, 4, 1, 3, 5)  # Fp12 = (a0, a1), a0 = w^0, w^2, w^4 and a1 = w^1, w^3, w^5


def f12_words(f):
    out = []
    for k in STRUCT_ORDER:
        out += words(f[k][0]) + words(f[k][1])
    return out


def f12_from_words(ws):
    f = [None] * 6
    for i, k in enumerate(STRUCT_ORDER):
        f[k] = (unwords(ws[24 * i:24 * i + 12]), unwords(ws[24 * i + 12:24 * i + 24]))
    return tuple(f)


def test_line_product_is_arrangement_independent():
    import torch
    subprocess.run(["make", "-s", "-C", HOST], check=True)
    probe = ctypes.CDLL(os.path.join(HOST, "libtower_probe.so"))
    rnd = random.Random(2024)
    n = 96
    fp2 = lambda: (rnd.randrange(PP.P), rnd.randrange(PP.P))
    fs = [tuple(fp2() for _ in range(6)) for _ in range(n)]
    ls = [(fp2(), fp2(), fp2()) for _ in range(n)]
    fs[0] = PP.ONE12
    ls[1] = ((PP.P - 1, PP.P - 1), (PP.P - 1, 0), (0, PP.P - 1))  # carries through every limb
    fw = np.array([f12_words(f) for f in fs], dtype=np.uint32)
    lw = np.array([words(c[0]) + words(c[1]) for l in ls for c in l], dtype=np.uint32).reshape(n, 72)
    exp = [PP.f12mul(f, (l[0], (0, 0), l[1], l[2], (0, 0), (0, 0))) for f, l in zip(fs, ls)]
    dl = torch.from_numpy(lw.view(np.int32)).cuda()
    for variant in (0, 1):
        df = torch.from_numpy(fw.view(np.int32).copy()).cuda()
        assert probe.tower_line(variant, ctypes.c_void_p(df.data_ptr()), ctypes.c_void_p(dl.data_ptr()), n) == 0
        got = df.cpu().numpy().view(np.uint32)
        bad = [i for i in range(n) if f12_from_words(got[i]) != exp[i]]
        assert not bad, (variant, bad[:8])
