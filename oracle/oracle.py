"""ctypes binding of the CPU oracle (oracle/liborc.so) -- TEST INFRASTRUCTURE.

The oracle restates the reference's FK20 algorithm on the CPU
(FK20Py/fk20_multi_cuda.py:67-246 and the files cited in fk20_oracle.c).  It is
imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and
reference arms, as the checker; the CUDA engine never calls it.

All arrays are numpy uint64 in the reference layout: fr_t = 4 limbs,
fp_t = 6 limbs, g1p_t = 18 limbs ({x, y, z}, homogeneous projective, standard
form, little-endian).  Points returned by the oracle are affine-normalised
({x, y, 1}, infinity (0, 1, 0)).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc.so")

P = 0x1A0111EA397FE69A4B1BA7B6434BACD764774B84F38512BF6730D2A0F6B0F6241EABFFFEB153FFFFB9FEFFFFFFFFAAAB
R = 0x73EDA753299D7D483339D80809A1D80553BDA402FFFE5BFEFFFFFFFF00000001

_lib = None


def build() -> None:
    """Compile liborc.so (gcc, portable flags)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        L.orc_init.restype = ctypes.c_int
        for name in ("orc_fp_op", "orc_fr_op", "orc_g1_op"):
            f = getattr(L, name)
            f.argtypes = [ctypes.c_int, u64p, u64p, u64p, ctypes.c_long]
            f.restype = ctypes.c_int
        L.orc_g1_is_point.argtypes = [u64p]
        L.orc_g1_generator.argtypes = [u64p]
        L.orc_root_of_unity.argtypes = [u64p, ctypes.c_uint]
        for name in ("orc_fr_fft", "orc_g1_fft"):
            f = getattr(L, name)
            f.argtypes = [u64p, u64p, ctypes.c_int, ctypes.c_long, ctypes.c_int]
        L.orc_seeded_fr.argtypes = [u64p, ctypes.c_uint64, ctypes.c_long]
        L.orc_setup.argtypes = [u64p, u64p, ctypes.c_long, ctypes.c_int]
        L.orc_xext_fft.argtypes = [u64p, u64p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_toeplitz.argtypes = [u64p, u64p, ctypes.c_int, ctypes.c_int]
        L.orc_fk20_row.argtypes = [u64p, ctypes.c_int, ctypes.c_int, u64p, u64p, u64p, u64p, u64p, u64p]
        L.orc_fk20_rows.argtypes = [u64p, u64p, ctypes.c_long, ctypes.c_int, ctypes.c_int, u64p, ctypes.c_int]
        L.orc_kzg_direct.argtypes = [u64p, u64p, ctypes.c_int, ctypes.c_int, u64p, ctypes.c_int, ctypes.c_int]
        L.orc_init()
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


# ---------------------------------------------------------------- int <-> limbs
def int_to_limbs(x: int, n: int) -> np.ndarray:
    return np.array([(x >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(n)], dtype=np.uint64)


def limbs_to_int(a) -> int:
    return sum(int(v) << (64 * i) for i, v in enumerate(np.asarray(a).reshape(-1)))


def ints_to_array(xs, n: int) -> np.ndarray:
    return np.stack([int_to_limbs(x, n) for x in xs]) if len(xs) else np.zeros((0, n), np.uint64)


# ---------------------------------------------------------------- element ops
FIELD_OPS = {"mul": 0, "sqr": 1, "add": 2, "sub": 3, "neg": 4, "inv": 5, "reduce": 6,
             "x2": 7, "x3": 8, "x4": 9, "x8": 10, "x12": 11}
G1_OPS = {"add": 0, "dbl": 1, "neg": 2, "sub": 3, "mul": 4, "normalize": 5}


def fp_op(op: str, a: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(-1, 6)
    if b is not None:
        b = np.ascontiguousarray(b, dtype=np.uint64).reshape(-1, 6)
    out = np.zeros_like(a)
    assert lib().orc_fp_op(FIELD_OPS[op], _p(out), _p(a), _p(b), a.shape[0]) == 0
    return out


def fr_op(op: str, a: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(-1, 4)
    if b is not None:
        b = np.ascontiguousarray(b, dtype=np.uint64).reshape(-1, 4)
    out = np.zeros_like(a)
    assert lib().orc_fr_op(FIELD_OPS[op], _p(out), _p(a), _p(b), a.shape[0]) == 0
    return out


def g1_op(op: str, a: np.ndarray, b: np.ndarray | None = None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(-1, 18)
    if b is not None:
        b = np.ascontiguousarray(b, dtype=np.uint64).reshape(a.shape[0], -1)
    out = np.zeros_like(a)
    assert lib().orc_g1_op(G1_OPS[op], _p(out), _p(a), _p(b), a.shape[0]) == 0
    return out


def g1_normalize(a: np.ndarray) -> np.ndarray:
    """Affine-normalise g1p_t points ({x, y, 1}, infinity (0,1,0)), canonical limbs."""
    shape = a.shape
    return g1_op("normalize", a).reshape(shape)


def g1_is_point(a: np.ndarray) -> bool:
    a = np.ascontiguousarray(a, dtype=np.uint64).reshape(18)
    return bool(lib().orc_g1_is_point(_p(a)))


def g1_generator() -> np.ndarray:
    out = np.zeros(18, np.uint64)
    lib().orc_g1_generator(_p(out))
    return out


def root_of_unity(order: int) -> int:
    out = np.zeros(4, np.uint64)
    lib().orc_root_of_unity(_p(out), order)
    return limbs_to_int(out)


def fr_fft(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    n = a.shape[-2]
    out = np.zeros_like(a)
    assert lib().orc_fr_fft(_p(out), _p(a), n, a.size // (4 * n), int(inverse)) == 0
    return out


def g1_fft(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    n = a.shape[-2]
    out = np.zeros_like(a)
    assert lib().orc_g1_fft(_p(out), _p(a), n, a.size // (18 * n), int(inverse)) == 0
    return out


# ---------------------------------------------------------------- seeded inputs
_GAMMA = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_R_LIMBS = int_to_limbs(R, 4)


def _splitmix(seed: int, idx: np.ndarray) -> np.ndarray:
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + (idx + np.uint64(1)) * _GAMMA
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def seeded_fr(seed: int, count: int) -> np.ndarray:
    """count uniform Fr values in [0, r): SplitMix64 stream of `seed`, 4 draws per
    candidate (limb 0..3), top limb masked to 63 bits, rejected if >= r.  Same
    stream as orc_seeded_fr in the C oracle."""
    out = []
    have = 0
    j0 = 0
    while have < count:
        need = int((count - have) * 1.12) + 64
        idx = np.arange(4 * j0, 4 * (j0 + need), dtype=np.uint64)
        v = _splitmix(seed, idx).reshape(need, 4)
        v[:, 3] &= np.uint64(0x7FFFFFFFFFFFFFFF)
        # lexicographic compare from the top limb: v < r
        lt = np.zeros(need, bool)
        eq = np.ones(need, bool)
        for k in (3, 2, 1, 0):
            lt |= eq & (v[:, k] < _R_LIMBS[k])
            eq &= v[:, k] == _R_LIMBS[k]
        acc = v[lt]
        out.append(acc[: count - have])
        have += min(len(acc), count - have)
        j0 += need
    return np.ascontiguousarray(np.concatenate(out)[:count])


def seeded_fr_c(seed: int, count: int) -> np.ndarray:
    out = np.zeros((count, 4), np.uint64)
    lib().orc_seeded_fr(_p(out), seed, count)
    return out


# ---------------------------------------------------------------- FK20
def setup(tau: np.ndarray, count: int, nthreads: int | None = None) -> np.ndarray:
    """s_i = tau^i G1 for i < count (affine g1p_t)."""
    out = np.zeros((count, 18), np.uint64)
    tau = np.ascontiguousarray(tau, dtype=np.uint64).reshape(4)
    lib().orc_setup(_p(out), _p(tau), count, nthreads or os.cpu_count() or 1)
    return out


def xext_fft(setup_pts: np.ndarray, n: int, l: int = 16, nthreads: int | None = None) -> np.ndarray:
    k = n // l
    assert setup_pts.shape[0] >= n - l
    out = np.zeros((l, 2 * k, 18), np.uint64)
    sp = np.ascontiguousarray(setup_pts, dtype=np.uint64)
    lib().orc_xext_fft(_p(out), _p(sp), n, l, nthreads or os.cpu_count() or 1)
    return out


def toeplitz(poly: np.ndarray, l: int = 16) -> np.ndarray:
    n = poly.shape[0]
    k = n // l
    out = np.zeros((l, 2 * k, 4), np.uint64)
    p = np.ascontiguousarray(poly, dtype=np.uint64)
    lib().orc_toeplitz(_p(out), _p(p), n, l)
    return out


def fk20_row(poly: np.ndarray, xext: np.ndarray, l: int = 16) -> dict:
    """All FK20 intermediates for one row: tc, tc_fft [l][2k] Fr; hext_fft, h,
    h_fft [2k] affine G1 (h's upper k entries are infinity)."""
    n = poly.shape[0]
    k = n // l
    m = 2 * k
    res = {
        "tc": np.zeros((l, m, 4), np.uint64),
        "tc_fft": np.zeros((l, m, 4), np.uint64),
        "hext_fft": np.zeros((m, 18), np.uint64),
        "h": np.zeros((m, 18), np.uint64),
        "h_fft": np.zeros((m, 18), np.uint64),
    }
    p = np.ascontiguousarray(poly, dtype=np.uint64)
    x = np.ascontiguousarray(xext, dtype=np.uint64)
    lib().orc_fk20_row(_p(p), n, l, _p(x), _p(res["tc"]), _p(res["tc_fft"]), _p(res["hext_fft"]),
                       _p(res["h"]), _p(res["h_fft"]))
    return res


def fk20_rows(polys: np.ndarray, xext: np.ndarray, l: int = 16, nthreads: int | None = None) -> np.ndarray:
    """h_fft[rows][2k] (affine) for rows x n polynomials, on nthreads host threads."""
    rows, n = polys.shape[0], polys.shape[1]
    m = 2 * (n // l)
    out = np.zeros((rows, m, 18), np.uint64)
    p = np.ascontiguousarray(polys, dtype=np.uint64)
    x = np.ascontiguousarray(xext, dtype=np.uint64)
    lib().orc_fk20_rows(_p(out), _p(p), rows, n, l, _p(x), nthreads or os.cpu_count() or 1)
    return out


def kzg_direct(poly: np.ndarray, tau: np.ndarray, l: int = 16, j0: int = 0, j1: int | None = None) -> np.ndarray:
    """Proofs j0..j1-1 of one row straight from the KZG definition with tau
    known: [q_j(tau)] G1, q_j = f div (X^l - w_2k^j)."""
    n = poly.shape[0]
    m = 2 * (n // l)
    j1 = m if j1 is None else j1
    out = np.zeros((j1 - j0, 18), np.uint64)
    p = np.ascontiguousarray(poly, dtype=np.uint64)
    t = np.ascontiguousarray(tau, dtype=np.uint64).reshape(4)
    lib().orc_kzg_direct(_p(out), _p(p), n, l, _p(t), j0, j1)
    return out


# ---------------------------------------------------------------- data-availability wire format
def g1_compress(a: np.ndarray) -> np.ndarray:
    """48-byte compressed encodings (count, 48) uint8 of g1p_t points: x as
    big-endian bytes with flags in the first byte -- 0x80 compressed, 0x40
    infinity (all else zero), 0x20 when y > (p - 1) / 2 -- the BLS12-381
    serialization of the ZCash/IETF convention (the format FK20Py's consumers
    read; py_ecc, which FK20Py imports, is absent here)."""
    pts = g1_normalize(np.ascontiguousarray(a, dtype=np.uint64).reshape(-1, 18))
    out = np.zeros((pts.shape[0], 48), np.uint8)
    for i, p in enumerate(pts):
        if limbs_to_int(p[12:18]) == 0:
            out[i, 0] = 0xC0
            continue
        x, y = limbs_to_int(p[0:6]), limbs_to_int(p[6:12])
        b = bytearray(x.to_bytes(48, "big"))
        b[0] |= 0x80 | (0x20 if y > (P - 1) // 2 else 0)
        out[i] = np.frombuffer(bytes(b), np.uint8)
    return out


def reverse_bit_order(rows: np.ndarray) -> np.ndarray:
    """Rows of a power-of-two length m, each permuted so that element i is the
    original element bitrev(i) (list_to_reverse_bit_order,
    FK20Py/kzg_proofs.py:105-118; the permutation is its own inverse)."""
    m = rows.shape[-2] if rows.ndim >= 2 else rows.shape[0]
    bits = m.bit_length() - 1
    idx = [int(format(i, f"0{bits}b")[::-1], 2) for i in range(m)]
    return rows[..., idx, :] if rows.ndim >= 2 else rows[idx]


def da_proofs(h_fft: np.ndarray) -> np.ndarray:
    """h_fft[rows][m] g1p_t -> proofs[rows][m][48] in data-availability order
    (FK20Py/fk20_multi_cuda.py:249-260)."""
    h = np.ascontiguousarray(h_fft, dtype=np.uint64)
    rows, m = h.shape[0], h.shape[1]
    comp = g1_compress(h.reshape(-1, 18)).reshape(rows, m, 48)
    return reverse_bit_order(comp)
