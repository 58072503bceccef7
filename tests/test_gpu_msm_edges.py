"""The MSM's exceptional mixed additions on the GPU (kernels_msm.cu g1z_madd):
the XYZZ accumulator equal to the added table entry (the doubling branch) and
equal to its negation (the infinity branch), reached by positive and by
negative signed digits, in both GLV passes (the s2 = s div lambda halves,
then phi, then the s1 = s mod lambda halves), and the addition that follows
an accumulator at infinity.  Random FK20 inputs never reach these branches;
here the bases xext_fft[i][c] are all the generator G except base 2, which
is -G, and the scalars are crafted per row, so the sums are known multiples
of G.  The reference's fk20_msm (fk20_msm.cu:23-66) uses complete formulas
and has no such branches: its result is the plain sum, which is what the
oracle gives."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

CB = 8  # table window of the context below: digits in [-128, 128], 17 windows per GLV half
LAMBDA = 0xAC45A4010001A40200000000FFFFFFFF  # phi = [lambda] on G1


def _scalar_rows(rows):
    """tc[row][i] for the 16 terms; rows 0..5 crafted, the rest seeded random."""
    s = np.zeros((rows, 16), dtype=object)
    s[:, :] = 0
    # 0: 2G, then 2G again: accumulator == entry -> doubling (4G)
    s[0, 0], s[0, 1] = 2, 2
    # 1: 4G, then 4 * (-G): accumulator == -entry -> infinity; then 5G from infinity
    s[1, 0], s[1, 1], s[1, 2], s[1, 3] = 2, 2, 4, 5
    # 2: 4G, then 252 = 2^8 - 4 on G: digit -4 (negated entry -4G) -> infinity, then digit 1 at window 1
    s[2, 0], s[2, 3] = 4, (1 << CB) - 4
    # 3: 4G, then 252 on -G: digit -4 gives +4G == accumulator -> doubling, then -256G
    s[3, 0], s[3, 2] = 4, (1 << CB) - 4
    # 4: the doubling branch on a top-window entry: 2^120 G (window 15, digit 1) twice
    s[4, 0], s[4, 1] = 1 << 120, 1 << 120
    # 5: all zero -> infinity
    # 6: the s2 pass: 2 lambda = 0 + 2 lambda twice -> doubling there, then phi
    s[6, 0], s[6, 1] = 2 * LAMBDA, 2 * LAMBDA
    # 7: the s2 pass: 2 lambda on G, then on -G -> infinity there
    s[7, 0], s[7, 2] = 2 * LAMBDA, 2 * LAMBDA
    rnd = O.seeded_fr(515, (rows - 8) * 16)
    for k in range(8, rows):
        for i in range(16):
            s[k, i] = O.limbs_to_int(rnd[(k - 8) * 16 + i])
    return s


def test_msm_exceptional_branches(engine):
    import torch
    n, rows = 1024, 32
    m = 2 * n // 16
    g = O.g1_generator()
    neg_g = O.g1_op("neg", g.reshape(1, 18))[0]
    xext = np.repeat(g.reshape(1, 1, 18), 16, 0).repeat(m, 1)
    xext[2, :] = neg_g
    sc = _scalar_rows(rows)
    tc = np.zeros((rows, 16, m, 4), np.uint64)
    for r in range(rows):
        for i in range(16):
            tc[r, i, :] = O.int_to_limbs(int(sc[r, i]) % O.R, 4)
    c = engine.Context(0, CB)
    try:
        c.load_xext_fft(n, engine.to_device(np.ascontiguousarray(xext)))
        hext = engine.empty((rows, m, 18))
        c.msm(hext, engine.to_device(tc), rows, n)
        torch.cuda.synchronize()
        got = O.g1_normalize(engine.to_host(hext).reshape(-1, 18)).reshape(rows, m, 18)
    finally:
        c.close()
    sign = [-1 if i == 2 else 1 for i in range(16)]
    ks = [sum(sign[i] * int(sc[r, i]) for i in range(16)) % O.R for r in range(rows)]
    assert ks[:8] == [4, 5, 256, (4 - 252) % O.R, 1 << 121, 0, 4 * LAMBDA % O.R, 0]
    exp = O.g1_normalize(O.g1_op("mul", np.repeat(g.reshape(1, 18), rows, 0), O.ints_to_array(ks, 4)))
    for r in range(rows):
        assert np.array_equal(got[r], np.repeat(exp[r:r + 1], m, 0)), r
