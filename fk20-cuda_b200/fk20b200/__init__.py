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
G2_OPS = {"add": 0, "dbl": 1, "neg": 2, "sub": 3, "mul": 4, "normalize": 5, "is_point": 6}

# every symbol declared in include/fk20_b200.h
ABI_SYMBOLS = (
    "fk20_ctx_create", "fk20_ctx_destroy", "fk20_ctx_load_xext_fft", "fk20_ctx_load_setup",
    "fk20_ctx_poly2h_fft", "fk20_ctx_poly2hext_fft", "fk20_ctx_msm", "fk20_ctx_batch",
    "fk20_ctx_device_bytes", "fk20_poly2h_fft", "fk20_poly2toeplitz_coefficients",
    "fk20_poly2toeplitz_coefficients_fft", "fk20_poly2hext_fft", "fk20_msm", "fk20_hext_fft2h_fft",
    "fk20_hext_fft2h", "fk20_hext_fft2hext", "fk20_h2h_fft", "fk20_hext2h", "fk20_setup2xext_fft",
    "fr_fft", "fr_ift", "g1p_fft", "g1p_ift", "fr_fft_n", "g1p_fft_n", "fp_op_n", "fr_op_n",
    "g1p_op_n", "fr_eq_n", "g1p_eq_n", "g1a_fromG1p_n", "fk20_bench_field", "fk20_version",
    "fk20_ctx_profile", "fk20_ctx_profile_read", "fk20_ctx_profile_read_executed", "fk20_program_cost", "fk20_bench_imad",
    "fk20_ctx_set", "fk20_ctx_status", "g1p_fft_noalloc", "fk20_ctx_get", "fk20_plan_create",
    "fk20_plan_launch", "fk20_plan_destroy", "fk20_ctx_autotune", "fk20_server_create", "fk20_server_submit",
    "fk20_server_wait", "fk20_server_get_stats", "fk20_server_reset_stats", "fk20_server_destroy",
    "fk20_g1p_compress_n", "fk20_h_fft2proofs", "fk20_ctx_poly2proofs", "fk20_ctx_batch_proofs",
    "fk20_ctx_load_commit", "fk20_ctx_commit", "fk20_pairing_check_n", "fk20_pairing_n", "g2p_op_n",
    "fk20_ctx_check_proof_multi", "fk20_default_release", "fk20_check_status", "fk20_server_cancel",
    "fk20_test_fail_allocations",
)

# kernel kinds of the per-launch profiler (FK20_K_* in the header)
KINDS = ("tc_fft", "msm", "stage_inv", "stage_fwd", "middle", "output", "fft_fused")
FK20_ETIMEOUT = 1005
FK20_ETOOBIG = 1006
FK20_EAGAIN = 1007
FK20_ECHECK = 1008
FK20_ECANCELED = 1009
FK20_OPT_FUSED_FFT = 1
FK20_OPT_MSM_THREADS = 2
FK20_OPT_FFT_BLOCKS_PER_SM = 3
FK20_OPT_WAIT_LIMIT = 4
FK20_OPT_TEST_UNPUBLISHED_TASK = 5
FK20_OPT_WINDOW = 6
FK20_OPT_TEST_CHECK = 7


class TuneResult(ctypes.Structure):
    _fields_ = [("window", ctypes.c_int), ("msm_threads", ctypes.c_int), ("fft_blocks_per_sm", ctypes.c_int),
                ("fused_fft", ctypes.c_int), ("ms", ctypes.c_float), ("ms_default", ctypes.c_float)]


class ServerConfig(ctypes.Structure):
    _fields_ = [("max_rows", ctypes.c_uint), ("slots", ctypes.c_uint), ("hbm_budget", ctypes.c_size_t),
                ("max_queue", ctypes.c_uint), ("fft_blocks_per_sm", ctypes.c_uint),
                ("latency_rows", ctypes.c_uint), ("burst_rows", ctypes.c_uint), ("engine", ctypes.c_uint),
                ("cohort_rows", ctypes.c_uint), ("cohorts", ctypes.c_uint), ("form_ms", ctypes.c_uint),
                ("stages_per_launch", ctypes.c_uint)]


class ServerStats(ctypes.Structure):
    _fields_ = [("requests", ctypes.c_uint64), ("proofs", ctypes.c_uint64), ("packs", ctypes.c_uint64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("wall_s", ctypes.c_double), ("proofs_per_s", ctypes.c_double),
                ("mean_pack_rows", ctypes.c_double), ("rejected", ctypes.c_uint64), ("nomem", ctypes.c_uint64),
                ("cancelled", ctypes.c_uint64),
                ("mean_wait_ms", ctypes.c_double), ("mean_enqueue_ms", ctypes.c_double),
                ("mean_run_ms", ctypes.c_double), ("mean_msm_ms", ctypes.c_double),
                ("mean_launch_ms", ctypes.c_double), ("launches", ctypes.c_uint64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


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
            "fk20_ctx_profile_read_executed": ([vp, i, ctypes.POINTER(ctypes.c_double)], i),
            "fk20_program_cost": ([i, ctypes.POINTER(i), ctypes.POINTER(i)], i),
            "fk20_bench_imad": ([vp, i, i, i, vp], i),
            "fk20_ctx_set": ([vp, i, i], i),
            "fk20_ctx_status": ([vp], i),
            "g1p_fft_noalloc": ([vp, vp, u, u, i, vp], i),
            "fk20_ctx_get": ([vp, i, ctypes.POINTER(i)], i),
            "fk20_plan_create": ([ctypes.POINTER(vp), vp, vp, vp, u, vp, vp, vp], i),
            "fk20_plan_launch": ([vp, vp], i),
            "fk20_plan_destroy": ([vp], i),
            "fk20_ctx_autotune": ([vp, u, u, sz, ctypes.POINTER(TuneResult), vp], i),
            "fk20_server_create": ([ctypes.POINTER(vp), vp, ctypes.POINTER(ServerConfig)], i),
            "fk20_server_submit": ([vp, vp, u, vp, ctypes.POINTER(ctypes.c_uint64)], i),
            "fk20_server_wait": ([vp, ctypes.c_uint64, i], i),
            "fk20_server_get_stats": ([vp, ctypes.POINTER(ServerStats)], i),
            "fk20_server_reset_stats": ([vp], i),
            "fk20_server_destroy": ([vp], i),
            "fk20_g1p_compress_n": ([vp, vp, sz, vp], i),
            "fk20_h_fft2proofs": ([vp, vp, u, u, vp], i),
            "fk20_ctx_poly2proofs": ([vp, vp, vp, u, u, vp], i),
            "fk20_ctx_batch_proofs": ([vp, vp, vp, u, vp, vp, vp, vp], i),
            "fk20_ctx_load_commit": ([vp, u, vp, i, vp], i),
            "fk20_ctx_commit": ([vp, vp, vp, u, u, vp], i),
            "fk20_pairing_check_n": ([vp, vp, vp, vp, vp, sz, vp], i),
            "fk20_ctx_check_proof_multi": ([vp, vp, vp, vp, vp, vp, u, vp, u, vp], i),
            "fk20_pairing_n": ([vp, vp, vp, sz, vp], i),
            "g2p_op_n": ([i, vp, vp, vp, sz, vp], i),
            "fk20_default_release": ([i], i),
            "fk20_check_status": ([ctypes.POINTER(i)], i),
            "fk20_server_cancel": ([vp, ctypes.c_uint64], i),
            "fk20_test_fail_allocations": ([i], i),
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

    def load_commit(self, n: int, setup, window: int = 0):
        call("fk20_ctx_load_commit", self.h, n, _ptr(setup), window, _stream())

    def commit(self, commitments, poly, rows: int, n: int):
        """commitments[rows] (g1p_t) = sum_i poly[row][i] * setup_i."""
        call("fk20_ctx_commit", self.h, _ptr(commitments), _ptr(poly), rows, n, _stream())

    def check_proof_multi(self, ok, commitments, proofs, x, ys, l: int, setup_g2, count: int):
        """ok[count] (uint8) = check_proof_multi of each (commitment, proof, x,
        ys[l]); setup_g2 = [s^k]G2 for k = 0..l (g2p_t rows).  Needs the
        commitment tables (load_commit with n >= 32)."""
        call("fk20_ctx_check_proof_multi", self.h, _ptr(ok), _ptr(commitments), _ptr(proofs), _ptr(x), _ptr(ys), l,
             _ptr(setup_g2), count, _stream())

    def poly2proofs(self, proofs, poly, rows: int, n: int):
        """proofs: uint8 CUDA tensor [rows][2n/16][48], data-availability order."""
        call("fk20_ctx_poly2proofs", self.h, _ptr(proofs), _ptr(poly), rows, n, _stream())

    def batch_proofs(self, proofs, polys, ns, poly_off, out_off):
        cnt = len(ns)
        call("fk20_ctx_batch_proofs", self.h, _ptr(proofs), _ptr(polys), cnt, (ctypes.c_uint * cnt)(*ns),
             (ctypes.c_size_t * cnt)(*poly_off), (ctypes.c_size_t * cnt)(*out_off), _stream())

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

    def get(self, option: int) -> int:
        v = ctypes.c_int()
        call("fk20_ctx_get", self.h, option, ctypes.byref(v))
        return v.value

    def autotune(self, n: int, rows: int = 128, max_table_bytes: int = 0) -> dict:
        r = TuneResult()
        call("fk20_ctx_autotune", self.h, n, rows, max_table_bytes, ctypes.byref(r), _stream())
        return {k: getattr(r, k) for k, _ in TuneResult._fields_}

    def status(self) -> int:
        return lib().fk20_ctx_status(self.h)

    def device_bytes(self) -> int:
        return lib().fk20_ctx_device_bytes(self.h)

    def profile(self, enable: bool = True):
        call("fk20_ctx_profile", self.h, int(enable))

    def profile_read(self) -> dict:
        """{kind: (ms, launches, products)} accumulated since profile(True);
        products are algorithmic limb products (fixed unit costs)."""
        out = {}
        for k, name in enumerate(KINDS):
            ms, n, pr = ctypes.c_double(), ctypes.c_long(), ctypes.c_double()
            call("fk20_ctx_profile_read", self.h, k, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(pr))
            out[name] = (ms.value, n.value, pr.value)
        return out

    def profile_read_executed(self) -> dict:
        """{kind: products} as executed by the kernels' formulas, same launches."""
        out = {}
        for k, name in enumerate(KINDS):
            pr = ctypes.c_double()
            call("fk20_ctx_profile_read_executed", self.h, k, ctypes.byref(pr))
            out[name] = pr.value
        return out


def version() -> str:
    return lib().fk20_version().decode()


def program_cost(index: int):
    """(doublings, additions) of fixed-scalar program `index` (w_512^index, or 2^-s at 512 + s)."""
    d, a = ctypes.c_int(), ctypes.c_int()
    call("fk20_program_cost", index, ctypes.byref(d), ctypes.byref(a))
    return d.value, a.value


# ------------------------------------------------------------------ batch plans (CUDA graphs)
class Plan:
    """A ragged batch layout bound to fixed device buffers, captured into a
    CUDA graph once; launch() replays it."""

    def __init__(self, ctx: Context, h_fft, polys, ns, poly_off, out_off):
        cnt = len(ns)
        h = ctypes.c_void_p()
        call("fk20_plan_create", ctypes.byref(h), ctx.h, _ptr(h_fft), _ptr(polys), cnt, (ctypes.c_uint * cnt)(*ns),
             (ctypes.c_size_t * cnt)(*poly_off), (ctypes.c_size_t * cnt)(*out_off))
        self.h = h
        self._keep = (ctx, h_fft, polys)

    def launch(self, stream=None):
        call("fk20_plan_launch", self.h, stream or _stream())

    def close(self):
        if self.h:
            call("fk20_plan_destroy", self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ request server
class Server:
    """Continuous-batching request server over a context (fk20_server_*).
    submit() takes HOST numpy arrays: the polynomial (n x 4 uint64) and the
    output (n/8 x 18 uint64); both are kept referenced until wait()."""

    def __init__(self, ctx: Context, max_rows: int = 0, slots: int = 0, hbm_budget: int = 0, max_queue: int = 0,
                 fft_blocks_per_sm: int = 0, latency_rows: int = 0, burst_rows: int = 0, engine: int = 0,
                 cohort_rows: int = 0, cohorts: int = 0, form_ms: int = 0, stages_per_launch: int = 0):
        cfg = ServerConfig(max_rows, slots, hbm_budget, max_queue, fft_blocks_per_sm, latency_rows, burst_rows,
                           engine, cohort_rows, cohorts, form_ms, stages_per_launch)
        h = ctypes.c_void_p()
        call("fk20_server_create", ctypes.byref(h), ctx.h, ctypes.byref(cfg))
        self.h = h
        self.ctx = ctx
        self._held = {}

    def submit(self, poly, out) -> int:
        n = poly.shape[0]
        t = ctypes.c_uint64()
        call("fk20_server_submit", self.h, ctypes.c_void_p(poly.ctypes.data), n, ctypes.c_void_p(out.ctypes.data),
             ctypes.byref(t))
        self._held[t.value] = (poly, out)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> int:
        rc = lib().fk20_server_wait(self.h, ticket, timeout_ms)
        if rc != FK20_EAGAIN:
            self._held.pop(ticket, None)
        return rc

    def cancel(self, ticket: int) -> int:
        """0: cancelled (the buffers are free again); FK20_EAGAIN: already on the GPU."""
        rc = lib().fk20_server_cancel(self.h, ticket)
        if rc == 0:
            self._held.pop(ticket, None)
        return rc

    def stats(self) -> dict:
        st = ServerStats()
        call("fk20_server_get_stats", self.h, ctypes.byref(st))
        return st.as_dict()

    def reset_stats(self):
        call("fk20_server_reset_stats", self.h)

    def close(self):
        if self.h:
            call("fk20_server_destroy", self.h)
            self.h = None
            self._held.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
