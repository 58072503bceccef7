"""Python binding of the B200 FK20 engine (libfk20b200.so) through its C ABI.

Thin ctypes layer over include/fk20_b200.h for tests, benchmarks and Python
callers.  Device buffers are torch CUDA tensors of dtype uint64 in the
reference layouts (fr_t = 4 limbs, g1p_t = 18 limbs, standard form); torch is
used only for device memory and streams.  Every call goes to the CUDA library:
if libfk20b200.so is missing or cannot load, import fails loudly -- there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libfk20b200.so")

FK20_OK = 0
FK20_EINVAL = 1001
FK20_ENOSETUP = 1002
FK20_ENOMEM = 1003
FK20_ENODEV = 1004

FIELD_OPS = {"mul": 0, "sqr": 1, "add": 2, "sub": 3, "neg": 4, "inv": 5, "reduce": 6,
             "x2": 7, "x3": 8, "x4": 9, "x8": 10, "x12": 11}
G1_OPS = {"add": 0, "dbl": 1, "neg": 2, "sub": 3, "mul": 4, "normalize": 5, "is_point": 6}

# every symbol declared in include/fk20_b200.h
ABI_SYMBOLS = (
    "fk20_ctx_create", "fk20_ctx_destroy", "fk20_ctx_load_xext_fft", "fk20_ctx_load_setup",
    "fk20_ctx_poly2h_fft", "fk20_ctx_poly2hext_fft", "fk20_ctx_msm", "fk20_ctx_batch",
    "fk20_ctx_device_bytes", "fk20_poly2h_fft", "fk20_poly2toeplitz_coefficients",
    "fk20_poly2toeplitz_coefficients_fft", "fk20_poly2hext_fft", "fk20_msm", "fk20_hext_fft2h_fft",
    "fk20_hext_fft2h", "fk20_hext_fft2hext", "fk20_h2h_fft", "fk20_hext2h", "fk20_setup2xext_fft",
    "fr_fft", "fr_ift", "g1p_fft", "g1p_ift", "fr_fft_n", "g1p_fft_n", "fp_op_n", "fr_op_n",
    "g1p_op_n", "fr_eq_n", "g1p_eq_n", "g1a_fromG1p_n", "fk20_bench_field", "fk20_version",
    "fk20_ctx_profile", "fk20_ctx_profile_read", "fk20_program_cost", "fk20_bench_imad",
    "fk20_ctx_set", "fk20_ctx_status", "g1p_fft_noalloc",
)

# kernel kinds of the per-launch profiler (FK20_K_* in the header)
KINDS = ("tc_fft", "msm", "stage_inv", "stage_fwd", "middle", "output", "fft_fused")
FK20_ETIMEOUT = 1005
FK20_ETOOBIG = 1006
FK20_OPT_FUSED_FFT = 1


class Fk20Error(RuntimeError):
    def __init__(self, name: str, code: int):
        super().__init__(f"{name} failed with code {code}")
        self.code = code


def build(jobs: int = 8) -> None:
    """Compile libfk20b200.so in-tree (nvcc, sm_100a)."""
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", PKG_DIR], check=True)


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}`")
        L = ctypes.CDLL(LIB_PATH)
        vp, u, sz, i = ctypes.c_void_p, ctypes.c_uint, ctypes.c_size_t, ctypes.c_int
        sig = {
            "fk20_ctx_create": ([ctypes.POINTER(vp), i, i], i),
            "fk20_ctx_destroy": ([vp], i),
            "fk20_ctx_load_xext_fft": ([vp, u, vp, vp], i),
            "fk20_ctx_load_setup": ([vp, u, vp, vp], i),
            "fk20_ctx_poly2h_fft": ([vp, vp, vp, u, u, vp], i),
            "fk20_ctx_poly2hext_fft": ([vp, vp, vp, u, u, vp], i),
            "fk20_ctx_msm": ([vp, vp, vp, u, u, vp], i),
            "fk20_ctx_batch": ([vp, vp, vp, u, vp, vp, vp, vp], i),
            "fk20_ctx_device_bytes": ([vp], sz),
            "fk20_poly2h_fft": ([vp, vp, vp, u], i),
            "fk20_poly2toeplitz_coefficients": ([vp, vp, u, vp], i),
            "fk20_poly2toeplitz_coefficients_fft": ([vp, vp, u, vp], i),
            "fk20_poly2hext_fft": ([vp, vp, vp, u, vp], i),
            "fk20_msm": ([vp, vp, vp, u, vp], i),
            "fk20_hext_fft2h_fft": ([vp, vp, u, vp], i),
            "fk20_hext_fft2h": ([vp, vp, u, vp], i),
            "fk20_hext_fft2hext": ([vp, vp, u, vp], i),
            "fk20_h2h_fft": ([vp, vp, u, vp], i),
            "fk20_hext2h": ([vp, u, vp], i),
            "fk20_setup2xext_fft": ([vp, vp, vp], i),
            "fr_fft": ([vp, vp, u, vp], i),
            "fr_ift": ([vp, vp, u, vp], i),
            "g1p_fft": ([vp, vp, u, vp], i),
            "g1p_ift": ([vp, vp, u, vp], i),
            "fr_fft_n": ([vp, vp, u, u, i, vp], i),
            "g1p_fft_n": ([vp, vp, u, u, i, vp], i),
            "fp_op_n": ([i, vp, vp, vp, sz, vp], i),
            "fr_op_n": ([i, vp, vp, vp, sz, vp], i),
            "g1p_op_n": ([i, vp, vp, vp, sz, vp], i),
            "fr_eq_n": ([vp, vp, vp, sz, vp], i),
            "g1p_eq_n": ([vp, vp, vp, sz, vp], i),
            "g1a_fromG1p_n": ([vp, vp, sz, vp], i),
            "fk20_bench_field": ([i, i, vp, sz, i, vp], i),
            "fk20_version": ([], ctypes.c_char_p),
            "fk20_ctx_profile": ([vp, i], i),
            "fk20_ctx_profile_read": ([vp, i, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_long),
                                       ctypes.POINTER(ctypes.c_double)], i),
            "fk20_program_cost": ([i, ctypes.POINTER(i), ctypes.POINTER(i)], i),
            "fk20_bench_imad": ([vp, i, i, i, vp], i),
            "fk20_ctx_set": ([vp, i, i], i),
            "fk20_ctx_status": ([vp], i),
            "g1p_fft_noalloc": ([vp, vp, u, u, i, vp], i),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def check(name: str, rc: int) -> None:
    if rc != 0:
        raise Fk20Error(name, rc)


def call(name: str, *args) -> None:
    check(name, getattr(lib(), name)(*args))


# ------------------------------------------------------------------ tensors
def to_device(a, device="cuda"):
    """numpy uint64 array -> torch uint64 CUDA tensor (same shape)."""
    import numpy as np
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64)).to(device)


def to_host(t):
    import torch
    return t.cpu().numpy() if isinstance(t, torch.Tensor) else t


def empty(shape, device="cuda"):
    import torch
    return torch.empty(shape, dtype=torch.uint64, device=device)


# ------------------------------------------------------------------ context
class Context:
    """A device context with fixed-base tables per polynomial length."""

    def __init__(self, device: int = 0, window: int = 0):
        h = ctypes.c_void_p()
        call("fk20_ctx_create", ctypes.byref(h), device, window)
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            call("fk20_ctx_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_xext_fft(self, n: int, xext_fft):
        call("fk20_ctx_load_xext_fft", self.h, n, _ptr(xext_fft), _stream())

    def load_setup(self, n: int, setup):
        call("fk20_ctx_load_setup", self.h, n, _ptr(setup), _stream())

    def poly2h_fft(self, h_fft, poly, rows: int, n: int, stream=None):
        call("fk20_ctx_poly2h_fft", self.h, _ptr(h_fft), _ptr(poly), rows, n, stream or _stream())

    def poly2hext_fft(self, hext_fft, poly, rows: int, n: int):
        call("fk20_ctx_poly2hext_fft", self.h, _ptr(hext_fft), _ptr(poly), rows, n, _stream())

    def msm(self, hext_fft, tc_fft, rows: int, n: int):
        call("fk20_ctx_msm", self.h, _ptr(hext_fft), _ptr(tc_fft), rows, n, _stream())

    def batch(self, h_fft, polys, ns, poly_off, out_off):
        import numpy as np
        cnt = len(ns)
        n_arr = (ctypes.c_uint * cnt)(*ns)
        po = (ctypes.c_size_t * cnt)(*poly_off)
        oo = (ctypes.c_size_t * cnt)(*out_off)
        call("fk20_ctx_batch", self.h, _ptr(h_fft), _ptr(polys), cnt, n_arr, po, oo, _stream())

    def set(self, option: int, value: int):
        call("fk20_ctx_set", self.h, option, value)

    def status(self) -> int:
        return lib().fk20_ctx_status(self.h)

    def device_bytes(self) -> int:
        return lib().fk20_ctx_device_bytes(self.h)

    def profile(self, enable: bool = True):
        call("fk20_ctx_profile", self.h, int(enable))

    def profile_read(self) -> dict:
        """{kind: (ms, launches, products)} accumulated since profile(True)."""
        out = {}
        for k, name in enumerate(KINDS):
            ms, n, pr = ctypes.c_double(), ctypes.c_long(), ctypes.c_double()
            call("fk20_ctx_profile_read", self.h, k, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(pr))
            out[name] = (ms.value, n.value, pr.value)
        return out


def version() -> str:
    return lib().fk20_version().decode()
