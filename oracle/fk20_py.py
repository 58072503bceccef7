"""Pure-Python restatement of FK20Py's data-availability multi-proof -- TEST INFRASTRUCTURE.

A line-by-line restatement of the reference's Python generator with plain
Python integers, written without py_ecc (which is absent here):
  fk20_multi_data_availability_optimized  FK20Py/fk20_multi_cuda.py:67-246
  toeplitz_part1 / part2 / part3          FK20Py/fk20_single.py:45-84
  fft / _fft / expand_root_of_unity       FK20Py/fft.py:17-55
  generate_setup, get_root_of_unity       FK20Py/kzg_proofs.py:22-44
The G1 group law is affine over y^2 = x^3 + 4 (g1p_ispoint.cu:34-60), with
None as the point at infinity.  Used on small sizes to cross-check the C
oracle; never on the product path.
"""
P = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB
MODULUS = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001
G1 = (0x17F1D3A73197D7942695638C4FA9AC0FC3688C4F9774B905A14E3A3F171BAC586C55E83FF97A1AEFFB3AF00ADB22C6BB,
      0x08B3F481E3AAA0F1A09E30ED741D8AE4FCF5E095D5D00AF600DB18CB2C04B3EDD03CC744A2888AE40CAA232946C5E7E1)
Z1 = None
PRIMITIVE_ROOT = 5


def add(a, b):
    if a is None:
        return b
    if b is None:
        return a
    x1, y1 = a
    x2, y2 = b
    if x1 == x2:
        if (y1 + y2) % P == 0:
            return None
        lam = 3 * x1 * x1 * pow(2 * y1, -1, P) % P
    else:
        lam = (y2 - y1) * pow(x2 - x1, -1, P) % P
    x3 = (lam * lam - x1 - x2) % P
    return x3, (lam * (x1 - x3) - y1) % P


def neg(a):
    return None if a is None else (a[0], (-a[1]) % P)


def multiply(pt, n):
    """double-and-add over the integer n (FK20Py calls py_ecc's multiply)."""
    acc = None
    for bit in bin(n % MODULUS)[2:] if n % MODULUS else "":
        acc = add(acc, acc)
        if bit == "1":
            acc = add(acc, pt)
    return acc


def get_root_of_unity(order):
    return pow(PRIMITIVE_ROOT, (MODULUS - 1) // order, MODULUS)


def generate_setup(s, size):
    return [multiply(G1, pow(s, i, MODULUS)) for i in range(size + 1)]


def _fft(vals, roots):
    if len(vals) == 1:
        return vals
    L = _fft(vals[::2], roots[::2])
    R = _fft(vals[1::2], roots[::2])
    o = [0] * len(vals)
    g1 = isinstance(vals[0], tuple) or vals[0] is None
    for i, (x, y) in enumerate(zip(L, R)):
        if g1:
            t = multiply(y, roots[i])
            o[i] = add(x, t)
            o[i + len(L)] = add(x, neg(t))
        else:
            t = y * roots[i]
            o[i] = (x + t) % MODULUS
            o[i + len(L)] = (x - t) % MODULUS
    return o


def fft(vals, root_of_unity, inv=False, g1=False):
    rootz = [1, root_of_unity]
    while rootz[-1] != 1:
        rootz.append(rootz[-1] * root_of_unity % MODULUS)
    if inv:
        invlen = pow(len(vals), MODULUS - 2, MODULUS)
        o = _fft(vals, rootz[:0:-1])
        return [multiply(x, invlen) for x in o] if g1 else [x * invlen % MODULUS for x in o]
    return _fft(vals, rootz[:-1])


def toeplitz_part1(x):
    xext = x + [Z1] * len(x)
    return fft(xext, get_root_of_unity(len(x) * 2), g1=True)


def toeplitz_part2(tc, xext_fft):
    tc_fft = fft(tc, get_root_of_unity(len(xext_fft)))
    return tc_fft, [multiply(v, w) for v, w in zip(xext_fft, tc_fft)]


def toeplitz_part3(hext_fft):
    return fft(hext_fft, get_root_of_unity(len(hext_fft)), inv=True, g1=True)[:len(hext_fft) // 2]


def fk20_da(polynomial, l, setup):
    """FK20Py fk20_multi_data_availability_optimized on `polynomial` (length n,
    the caller's un-extended polynomial): returns dict of intermediates."""
    n = len(polynomial)
    k = n // l
    xext_fft = []
    for i in range(l):
        x = setup[n - l - 1 - i::-l] + [Z1]
        xext_fft.append(toeplitz_part1(x))
    hext_fft = [Z1] * 2 * k
    tcs, tcffts = [], []
    for i in range(l):
        tc = polynomial[-i - 1::l] + [0] * (k + 1) + polynomial[2 * l - i - 1:-l - i:l]
        tc_fft, part = toeplitz_part2(tc, xext_fft[i])
        tcs.append(tc)
        tcffts.append(tc_fft)
        hext_fft = [add(v, w) for v, w in zip(hext_fft, part)]
    h = toeplitz_part3(hext_fft) + [Z1] * k
    h_fft = fft(h, get_root_of_unity(2 * k), g1=True)
    return {"xext_fft": xext_fft, "tc": tcs, "tc_fft": tcffts, "hext_fft": hext_fft, "h": h, "h_fft": h_fft}
