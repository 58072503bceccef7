"""Golden FK20 vectors from the reference's own CUDA kernels, run on a B200.

The reference's FK20 test vectors are not in its tree (fk20_testvector.cu is
listed in .MISSING_LARGE_BLOBS, test.tar.xz is an LFS pointer) and its Python
generator needs py_ecc, which is absent.  This script regenerates them from
the reference itself: the unmodified reference library built by
oracle/ref/Makefile (oracle/_ref/libfk20ref.so) runs its six-launch pipeline
(fk20_poly2h_fft.cu:57-77) on seeded inputs, and every intermediate is
recorded as a SHA-256 of its canonical affine bytes, plus a few literal points.

Inputs (same generators as the tests): tau = seeded_fr(424242, 1), setup
s_i = tau^i G1 and xext_fft from the oracle, polynomial rows
seeded_fr(777, rows * 4096).  Run on a GPU box:
    python tests/golden/make_ref_gpu_fixtures.py
"""
import ctypes
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "fk20-cuda_b200"))
import oracle as O  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "reference_fk20_pin.json")
ROWS, N, TAU_SEED, POLY_SEED = 2, 4096, 424242, 777


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u8").tobytes()).hexdigest()


def canon_fr(a):
    return O.fr_op("reduce", a.reshape(-1, 4)).reshape(a.shape)


def canon_g1(a):
    return O.g1_normalize(a.reshape(-1, 18)).reshape(a.shape)


def reference_run(poly, xext):
    import torch
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libfk20ref.so"), mode=os.RTLD_LOCAL)
    rows = poly.shape[0]
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64)).cuda()
    dpoly, dxext = dev(poly), dev(xext)
    tc = torch.zeros((rows, 16, 512, 4), dtype=torch.uint64, device="cuda")
    tcf = torch.zeros_like(tc)
    hext = torch.zeros((rows, 512, 18), dtype=torch.uint64, device="cuda")
    h, hf = torch.zeros_like(hext), torch.zeros_like(hext)
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = lib.ref_fk20_stages(P(dpoly), P(dxext), ctypes.c_uint(rows), P(tc), P(tcf), P(hext), P(h), P(hf))
    assert rc == 0, rc
    return {k: v.cpu().numpy() for k, v in dict(tc=tc, tc_fft=tcf, hext_fft=hext, h=h, h_fft=hf).items()}


def main():
    tau = O.seeded_fr(TAU_SEED, 1)[0]
    setup = O.setup(tau, N + 1)
    xext = O.xext_fft(setup, N, 16)
    poly = O.seeded_fr(POLY_SEED, ROWS * N).reshape(ROWS, N, 4)
    ref = reference_run(poly, xext)
    canon = {"tc": canon_fr(ref["tc"]), "tc_fft": canon_fr(ref["tc_fft"]),
             "hext_fft": canon_g1(ref["hext_fft"]), "h": canon_g1(ref["h"]), "h_fft": canon_g1(ref["h_fft"])}
    data = {
        "source": "lCardosoSantos/FK20-CUDA kernels (fk20_poly2h_fft.cu:57-77) compiled for sm_100a, run on B200",
        "inputs": {"rows": ROWS, "n": N, "l": 16, "tau_seed": TAU_SEED, "poly_seed": POLY_SEED,
                   "xext_fft_sha256": digest(xext)},
        "sha256": {k: [digest(v[r]) for r in range(ROWS)] for k, v in canon.items()},
        "h_fft_row0_first": [[hex(O.limbs_to_int(p[0:6])), hex(O.limbs_to_int(p[6:12]))] for p in canon["h_fft"][0][:4]],
    }
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
