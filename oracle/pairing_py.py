"""BLS12-381 pairing restated in pure Python -- TEST INFRASTRUCTURE.

The reference verifies multiproofs with py_ecc's pairing (check_proof_multi,
FK20Py/kzg_proofs.py:207-232); py_ecc is absent here, so this restates the
published optimal-ate construction for BLS12 curves in its plainest form, as
the checker of the engine's CUDA pairing (csrc/kernels_pairing.cu), which
computes the same values by other means (tower arithmetic, projective lines,
the split final exponentiation): after the final exponentiation they agree
exactly, as the Miller values differ only by factors in proper subfields.

  * Fp2 = Fp[u]/(u^2 + 1); Fp12 = Fp2[w]/(w^6 - xi), xi = 1 + u, elements as
    6 coefficients of w.
  * G2 on the M-type twist E': y^2 = x^3 + 4 xi; psi(x', y') = (x'/w^2, y'/w^3)
    maps it into E(Fp12).
  * Miller loop over the bits of |z| = 0xd201000000010000 with affine T; the
    line through T with twist slope L, evaluated at P and scaled by w^3:
    (L xT - yT) + (-L xP) w^2 + yP w^3 (the factor w^3 and the vertical lines
    vanish in the final exponentiation).
  * Final exponentiation by 3 (p^12 - 1)/r as one plain exponent (the cube is
    what the standard decomposition of the hard part computes; a fixed power
    coprime to r keeps the pairing non-degenerate and bilinear).

Because z < 0 and the loop runs over |z|, the value is e(P, Q)^-1 for the
usual normalisation: a non-degenerate bilinear pairing all the same, which is
all a verification equation needs.
"""
P = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB
R = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
Z_ABS = 0xD201000000010000
FINAL_EXP = 3 * ((P ** 12 - 1) // R)
G2_X = (0x024AA2B2F08F0A91260805272DC51051C6E47AD4FA403B02B4510B647AE3D1770BAC0326A805BBEFD48056C8C121BDB8,
        0x13E02B6052719F607DACD3A088274F65596BD0D09920B61AB5DA61BBDC7F5049334CF11213945D57E5AC7D055D042B7E)
G2_Y = (0x0CE5D527727D6E118CC9CDC6DA2E351AADFD9BAA8CBDD3A76D429A695160D12C923AC9CC3BACA289E193548608B82801,
        0x0606C4A02EA734CC32ACD2B02BC28B99CB3E287E85A763AF267492AB572E99AB3F370D275CEC1DA1AAA9075FF05F79BE)
B2 = (4, 4)  # 4 xi


# ---------------------------------------------------------------- Fp2
def f2add(a, b): return ((a[0] + b[0]) % P, (a[1] + b[1]) % P)
def f2sub(a, b): return ((a[0] - b[0]) % P, (a[1] - b[1]) % P)
def f2neg(a): return ((-a[0]) % P, (-a[1]) % P)
def f2mul(a, b): return ((a[0] * b[0] - a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)
def f2xi(a): return ((a[0] - a[1]) % P, (a[0] + a[1]) % P)  # a (1 + u)


def f2inv(a):
    ni = pow((a[0] * a[0] + a[1] * a[1]) % P, P - 2, P)
    return (a[0] * ni % P, (-a[1]) * ni % P)


# ---------------------------------------------------------------- Fp12 (6 Fp2 coefficients of w)
ONE12 = ((1, 0), (0, 0), (0, 0), (0, 0), (0, 0), (0, 0))


def f12mul(a, b):
    t = [(0, 0)] * 11
    for i in range(6):
        for j in range(6):
            t[i + j] = f2add(t[i + j], f2mul(a[i], b[j]))
    return tuple(f2add(t[k], f2xi(t[k + 6])) if k + 6 < 11 else t[k] for k in range(6))


def f12pow(a, e):
    r = ONE12
    for bit in bin(e)[2:]:
        r = f12mul(r, r)
        if bit == "1":
            r = f12mul(r, a)
    return r


# ---------------------------------------------------------------- G2 (affine, twist)
def g2add(p, q):
    if p is None:
        return q
    if q is None:
        return p
    if p[0] == q[0]:
        if f2add(p[1], q[1]) == (0, 0):
            return None
        lam = f2mul(f2mul((3, 0), f2mul(p[0], p[0])), f2inv(f2add(p[1], p[1])))
    else:
        lam = f2mul(f2sub(q[1], p[1]), f2inv(f2sub(q[0], p[0])))
    x3 = f2sub(f2sub(f2mul(lam, lam), p[0]), q[0])
    return (x3, f2sub(f2mul(lam, f2sub(p[0], x3)), p[1]))


def g2mul(k, q):
    r = None
    for bit in bin(k)[2:]:
        r = g2add(r, r)
        if bit == "1":
            r = g2add(r, q)
    return r


def g2_generator():
    return (G2_X, G2_Y)


# ---------------------------------------------------------------- pairing
def _line(lam, t, xp, yp):
    c0 = f2sub(f2mul(lam, t[0]), t[1])
    c1 = f2neg(f2mul(lam, (xp, 0)))
    return (c0, (0, 0), c1, (yp, 0), (0, 0), (0, 0))


def miller(p, q):
    """p = (x, y) affine over Fp, q affine over Fp2 (both not infinity)."""
    xp, yp = p
    f, t = ONE12, q
    for bit in bin(Z_ABS)[3:]:
        lam = f2mul(f2mul((3, 0), f2mul(t[0], t[0])), f2inv(f2add(t[1], t[1])))
        f = f12mul(f12mul(f, f), _line(lam, t, xp, yp))
        x3 = f2sub(f2mul(lam, lam), f2add(t[0], t[0]))
        t = (x3, f2sub(f2mul(lam, f2sub(t[0], x3)), t[1]))
        if bit == "1":
            lam = f2mul(f2sub(q[1], t[1]), f2inv(f2sub(q[0], t[0])))
            f = f12mul(f, _line(lam, t, xp, yp))
            x3 = f2sub(f2sub(f2mul(lam, lam), t[0]), q[0])
            t = (x3, f2sub(f2mul(lam, f2sub(t[0], x3)), t[1]))
    return f


def pairing(p, q):
    """e(p, q) as 6 Fp2 coefficients; p, q affine or None (infinity)."""
    if p is None or q is None:
        return ONE12
    return f12pow(miller(p, q), FINAL_EXP)


def pairing_check(p1, q1, p2, q2) -> bool:
    """e(p1, q1) == e(p2, q2), with one final exponentiation."""
    f = ONE12
    if p1 is not None and q1 is not None:
        f = f12mul(f, miller(p1, q1))
    if p2 is not None and q2 is not None:
        f = f12mul(f, miller((p2[0], (-p2[1]) % P), q2))
    return f12pow(f, FINAL_EXP) == ONE12


# ---------------------------------------------------------------- G1 (affine over Fp) and check_proof_multi
def g1add(p, q):
    if p is None:
        return q
    if q is None:
        return p
    if p[0] == q[0]:
        if (p[1] + q[1]) % P == 0:
            return None
        lam = 3 * p[0] * p[0] * pow(2 * p[1], P - 2, P) % P
    else:
        lam = (q[1] - p[1]) * pow(q[0] - p[0], P - 2, P) % P
    x3 = (lam * lam - p[0] - q[0]) % P
    return (x3, (lam * (p[0] - x3) - p[1]) % P)


def g1mul(k, p):
    r = None
    for bit in bin(k % R)[2:]:
        r = g1add(r, r)
        if bit == "1":
            r = g1add(r, p)
    return r


def g1neg(p):
    return None if p is None else (p[0], (-p[1]) % P)


def check_proof_multi(commitment, proof, x, ys, setup_g1, setup_g2):
    """FK20Py/kzg_proofs.py:207-232: the proof that f(x w^i) = ys[i], i < n
    (w the n-th root of unity 5^((r-1)/n)), for the polynomial committed in
    `commitment`; setup_g1 / setup_g2 = [s^k]G1 / [s^k]G2.  Affine points
    (None = infinity), field elements as ints."""
    n = len(ys)
    w = pow(5, (R - 1) // n, R)
    inv_n, inv_x = pow(n, R - 2, R), pow(x, R - 2, R)
    # interpolation over the coset: inverse DFT of ys, then coefficient i / x^i
    interp = [sum(ys[k] * pow(w, (R - 1 - j * k) % (R - 1), R) for k in range(n)) * inv_n % R for j in range(n)]
    interp = [c * pow(inv_x, i, R) % R for i, c in enumerate(interp)]
    xn_minus_yn = g2add(setup_g2[n], g2mul((R - pow(x, n, R)) % R, setup_g2[0]))
    lincomb = None
    for pt, c in zip(setup_g1, interp):
        lincomb = g1add(lincomb, g1mul(c, pt))
    com_minus_interp = g1add(commitment, g1neg(lincomb))
    # e(C - I(s), G2) == e(proof, [s^n - x^n]G2)
    return pairing_check(com_minus_interp, setup_g2[0], proof, xn_minus_yn)
