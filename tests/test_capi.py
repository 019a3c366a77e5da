"""The C-ABI library loads and exports every symbol include/*.h declares
(no compute call here: these run on machines without a GPU)."""
import ctypes
import glob
import os
import re

from sparkit_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(sk_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header():
    bound = {name for name, _ in _lib.SIGNATURES}
    assert declared_functions() <= bound | set()


def test_version_and_device_count():
    L = _lib.lib()
    assert b"sm_100a" in L.sk_version()
    n = ctypes.c_int(-1)
    assert L.sk_device_count(ctypes.byref(n)) == 0
    assert n.value >= 0


def test_no_device_is_reported_not_faked():
    """Without a GPU the library refuses to create handles (no CPU path)."""
    L = _lib.lib()
    n = ctypes.c_int(0)
    L.sk_device_count(ctypes.byref(n))
    if n.value > 0:
        return
    import numpy as np
    rp = np.array([0, 1], np.int64)
    ci = np.array([0], np.int64)
    v = np.array([1.0])
    h = ctypes.c_void_p()
    st = L.sk_csr_create(ctypes.byref(h), 1, 1, rp.ctypes.data_as(ctypes.c_void_p),
                         ci.ctypes.data_as(ctypes.c_void_p), v.ctypes.data_as(ctypes.c_void_p), 0)
    assert st == 10  # SK_NO_DEVICE
    assert b"device" in L.sk_last_error()


def test_built_for_sm100a_only():
    """The build recipe targets sm_100a and nothing else."""
    from sparkit_b200 import build
    flags = " ".join(build.NVCC_FLAGS)
    assert "arch=compute_100a,code=sm_100a" in flags
    assert "compute_90" not in flags and "sm_90" not in flags
