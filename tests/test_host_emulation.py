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


def fused_schedule(emul, G, log_m):
    nseg = len(G)
    cap = sum(g * (1 << l) // 2 * (2 * l - 1) for g, l in zip(G, log_m))
    out = np.zeros((cap, 7), np.int32)
    ga, la = (ctypes.c_int * nseg)(*G), (ctypes.c_int * nseg)(*log_m)
    n = emul.emul_fused_schedule(nseg, ga, la, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.c_long(cap))
    assert n == cap
    return out


@pytest.mark.parametrize("G,log_m", [([1], [9]), ([3, 2, 5], [9, 8, 7]), ([1, 1, 1, 2], [7, 9, 7, 8])])
def test_fused_fft_schedule(emul, G, log_m):
    """The persistent launch's task order (csrc/fused_plan.cuh, decoded the way
    the kernel decodes it): every stage of every segment touches each position
    of each row group exactly once, every task only depends on tasks of lower
    index (so the bounded waits always end), and running the butterflies in
    task order on Fr values gives FFT(upper half zeroed(IFFT without 1/m)) per
    segment -- the hext_fft -> h_fft map of the pipeline."""
    emul.emul_fused_schedule.restype = ctypes.c_long
    sched = fused_schedule(emul, G, log_m)
    R = O.R
    w512 = O.root_of_unity(512)
    rng = np.random.default_rng(7)
    vals = {}
    for k, (g_cnt, L) in enumerate(zip(G, log_m)):
        for g in range(g_cnt):
            vals[(k, g)] = [int(x) % R for x in rng.integers(0, 2**62, 1 << L)]
    start = {key: list(v) for key, v in vals.items()}
    last_writer = {}  # (seg, g, pos) -> (stage, task index)
    seen = set()
    for t, (seg, S, g, i0, i1, tix, kind) in enumerate(sched.tolist()):
        for p in (i0, i1):
            key = (seg, S, g, p)
            assert key not in seen
            seen.add(key)
            if S > 0:
                st, idx = last_writer[(seg, g, p)]
                assert st == S - 1 and idx < t
            last_writer[(seg, g, p)] = (S, t)
        v = vals[(seg, g)]
        wt = pow(w512, tix, R)
        u, x = v[i0], v[i1]
        if kind == 0:
            v[i0], v[i1] = (u + x) % R, (u - x) * wt % R
        elif kind == 2:
            v[i0] = v[i1] = (u + x) % R
        else:
            x = x * wt % R
            v[i0], v[i1] = (u + x) % R, (u - x) % R
    for k, (g_cnt, L) in enumerate(zip(G, log_m)):
        m = 1 << L
        assert len([s for s in seen if s[0] == k]) == g_cnt * m * (2 * L - 1)
        wp = [pow(w512, (512 // m) * e, R) for e in range(m)]  # powers of w_m
        for g in range(g_cnt):
            x = start[(k, g)]
            inv = [sum(x[j] * wp[(-i * j) % m] for j in range(m)) % R for i in range(m)]
            inv[m // 2:] = [0] * (m // 2)
            fwd = [sum(inv[j] * wp[(i * j) % m] for j in range(m)) % R for i in range(m)]
            assert vals[(k, g)] == fwd, (k, g)


def test_fused_fft_schedule_in_stage_windows(emul):
    """The server's cohort engine runs each segment's 17 (15, 13) stages over
    several launches, each launch a stage window per segment, windows of
    different segments starting at different stages.  Replayed launch by
    launch on Fr values: inside a launch every task depends only on tasks of
    lower index or on an earlier launch, the task order keeps windows of
    different segments side by side (relative stage first), and the result
    is FFT(upper half zeroed(IFFT)) per segment, as with one launch."""
    f = emul.emul_fused_schedule_w
    f.restype = ctypes.c_long
    R = O.R
    w512 = O.root_of_unity(512)
    rng = np.random.default_rng(9)
    G, log_m = [1, 2, 1], [9, 8, 7]
    total = [2 * l - 1 for l in log_m]
    # staggered windows: segment k starts k launches late, 3 stages a launch
    vals = {(k, g): [int(x) % R for x in rng.integers(0, 2**62, 1 << L)]
            for k, (gc, L) in enumerate(zip(G, log_m)) for g in range(gc)}
    start = {key: list(v) for key, v in vals.items()}
    done = [-3 * k for k in range(3)]  # stages run so far (negative: not started)
    launches = 0
    while any(d < t for d, t in zip(done, total)):
        segs = [k for k in range(3) if 0 <= done[k] < total[k]]
        lo = [done[k] for k in segs]
        hi = [min(total[k], done[k] + 3) for k in segs]
        if segs:
            nseg = len(segs)
            cap = sum(G[k] * (1 << log_m[k]) // 2 * (h - l) for k, l, h in zip(segs, lo, hi))
            out = np.zeros((cap, 7), np.int32)
            ci = lambda a: (ctypes.c_int * nseg)(*a)
            n = f(nseg, ci([G[k] for k in segs]), ci([log_m[k] for k in segs]), ci(lo), ci(hi),
                  out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ctypes.c_long(cap))
            assert n == cap
            writer = {}
            rel_prev = -1
            for t, (j, S, g, i0, i1, tix, kind) in enumerate(out.tolist()):
                k = segs[j]
                rel = S - lo[j]
                assert lo[j] <= S < hi[j] and rel >= rel_prev  # relative stage never goes back
                rel_prev = rel
                for p in (i0, i1):
                    if S > lo[j]:  # produced in this launch by the previous stage, at a lower index
                        st, idx = writer[(k, g, p)]
                        assert st == S - 1 and idx < t
                    writer[(k, g, p)] = (S, t)
                v = vals[(k, g)]
                wt = pow(w512, tix, R)
                u, x = v[i0], v[i1]
                if kind == 0:
                    v[i0], v[i1] = (u + x) % R, (u - x) * wt % R
                elif kind == 2:
                    v[i0] = v[i1] = (u + x) % R
                else:
                    x = x * wt % R
                    v[i0], v[i1] = (u + x) % R, (u - x) % R
            for j, k in enumerate(segs):
                done[k] = hi[j]
        for k in range(3):
            if done[k] < 0:
                done[k] += 3 if done[k] < 0 else 0
        launches += 1
    assert launches >= 7
    for k, (g_cnt, L) in enumerate(zip(G, log_m)):
        m = 1 << L
        wp = [pow(w512, (512 // m) * e, R) for e in range(m)]
        for g in range(g_cnt):
            x = start[(k, g)]
            inv = [sum(x[j] * wp[(-i * j) % m] for j in range(m)) % R for i in range(m)]
            inv[m // 2:] = [0] * (m // 2)
            fwd = [sum(inv[j] * wp[(i * j) % m] for j in range(m)) % R for i in range(m)]
            assert vals[(k, g)] == fwd, (k, g)


LAMBDA = 0xAC45A4010001A40200000000FFFFFFFF  # phi = [lambda] on G1, lambda^2 + lambda + 1 = r


def program_partial_sums(prog):
    """Replays a twiddle program (scalar_prog.cuh) on scalars mod r: yields,
    before every mixed addition, (accumulator scalar, added point's scalar),
    and returns the scalar of the result."""
    r = O.R
    hdr = int(prog[0])
    assert not hdr & 0x300
    top, acc, started, adds = hdr & 0xFF, 0, False, []
    for pos in range(top, -1, -1):
        if started:
            acc = 2 * acc % r
        byte = (int(prog[1 + (pos >> 2)]) >> ((pos & 3) * 8)) & 0xFF
        for h in (0, 1):
            code = (byte >> (4 * h)) & 15
            if code & 1:
                d = (2 * (code >> 2) + 1) * (-1 if code & 2 else 1)
                q = d * (LAMBDA if h else 1) % r
                if started:
                    adds.append((acc, q))
                    acc = (acc + q) % r
                else:
                    acc = q
                started = True
    if hdr & 0x400:
        acc = -acc % r
    return adds, acc


def test_programs_avoid_the_mixed_additions_exceptional_cases(emul):
    """The programs' main loop adds table points with the Jacobian mixed
    addition, which is wrong when the accumulator equals the added point or
    its negative, or is infinity.  For a point P of prime order r, acc = [a]P
    and Q = [q]P, so this happens exactly when a = +-q or a = 0 (mod r): checked
    here for every program the library builds (w^t, t < 512, w the 512th root
    of unity of the twiddles, and 2^-s, s < 16), and each program's result is
    its scalar."""
    r = O.R
    w = O.root_of_unity(512)
    scalars = [pow(w, t, r) for t in range(512)] + [pow(pow(2, s, r), r - 2, r) for s in range(16)]
    prog = np.zeros(64, np.uint32)
    checked = 0
    for k in scalars:
        emul.emul_make_program(prog.ctypes.data_as(ctypes.c_void_p), P(O.int_to_limbs(k, 4)))
        if int(prog[0]) & 0x300:  # 0 or +-1: no arithmetic
            assert k in (1, r - 1)
            continue
        adds, res = program_partial_sums(prog)
        assert res == k
        for a, q in adds:
            assert a != 0 and a != q and a != (r - q) % r, (hex(k), hex(a), hex(q))
        checked += len(adds)
    assert checked > 20000


def test_glv_split_of_msm_scalars(emul):
    """The MSM's scalar split (csrc/glv.cuh): s = s1 + s2 lambda with
    s1 = s mod lambda and s2 = s div lambda, both below 2^128, for random
    scalars below r and for the edges of the Barrett estimate."""
    r = O.R
    rng = np.random.default_rng(12)
    xs = [int.from_bytes(rng.bytes(32), "little") % r for _ in range(4000)]
    xs += [0, 1, LAMBDA - 1, LAMBDA, LAMBDA + 1, 2 * LAMBDA - 1, 2 * LAMBDA, r - 1, r - 2, r - LAMBDA,
           LAMBDA * LAMBDA, LAMBDA * LAMBDA - 1, (1 << 255) - 1, (1 << 254), (1 << 128) - 1, 1 << 128]
    s = O.ints_to_array(xs, 4)
    out = np.zeros((len(xs), 8), np.uint64)
    emul.emul_glv_split(P(out), P(s), len(xs))
    for j, x in enumerate(xs):
        s1, s2 = O.limbs_to_int(out[j, :4]), O.limbs_to_int(out[j, 4:])
        assert (s1, s2) == (x % LAMBDA, x // LAMBDA), hex(x)
        assert s1 < 1 << 128 and s2 < 1 << 128
