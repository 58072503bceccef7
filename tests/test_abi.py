"""The C-ABI library: every symbol declared in include/fk20_b200.h is exported
by libfk20b200.so (no GPU needed: only loading and symbol lookup)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fk20_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*([A-Za-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_parses():
    names = declared_functions()
    assert "fk20_poly2h_fft" in names and "g1p_fft" in names and len(names) >= 30


def test_library_exports_every_declared_symbol():
    import fk20b200
    if not os.path.exists(fk20b200.LIB_PATH):
        pytest.skip("libfk20b200.so not built (run __graft_entry__.build())")
    L = ctypes.CDLL(fk20b200.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, missing
    assert set(declared_functions()) == set(fk20b200.ABI_SYMBOLS)


def test_version_string_without_gpu():
    import fk20b200
    if not os.path.exists(fk20b200.LIB_PATH):
        pytest.skip("libfk20b200.so not built")
    assert fk20b200.version().startswith("fk20-b200")


def test_no_device_is_reported_not_faked():
    """Without a GPU the engine refuses work with FK20_ENODEV instead of
    computing anything on the CPU."""
    import torch
    import fk20b200
    if torch.cuda.is_available() or not os.path.exists(fk20b200.LIB_PATH):
        pytest.skip("only meaningful on a machine without a GPU")
    h = ctypes.c_void_p()
    rc = fk20b200.lib().fk20_ctx_create(ctypes.byref(h), 0, 0)
    assert rc == fk20b200.FK20_ENODEV
