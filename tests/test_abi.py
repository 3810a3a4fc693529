"""The C-ABI library loads and exports every symbol include/jfem_gpu.h declares (no compute)."""
import ctypes
import os
import re

from jfem_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    with open(os.path.join(ROOT, "include", "jfem_gpu.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jfg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_header():
    lib = ctypes.CDLL(N.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(N.EXPORTED)


def test_version_and_no_device_error():
    L = N.load()
    assert b"sm_100a" in L.jfg_version()
    h = ctypes.c_void_p()
    st = L.jfg_create(10**6, ctypes.byref(h))
    assert st in (N.ERR_NO_DEVICE, N.ERR_BAD_ARG)
