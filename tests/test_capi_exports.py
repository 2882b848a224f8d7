"""CPU checks of the C-ABI library: it loads without a GPU and exports every
entry point that include/mpsgpu.h declares (no compute call is made)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "mpsdyn_b200", "libmpsgpu.so")


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "mpsgpu.h")).read()
    return sorted(set(re.findall(r"\b(mpsgpu_[a-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        from mpsdyn_b200 import build
        build.build()
    return ctypes.CDLL(LIB)


def test_every_declared_symbol_is_exported(lib):
    syms = declared_symbols()
    assert len(syms) >= 25
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    from mpsdyn_b200 import capi
    assert sorted(capi.EXPORTS) == declared_symbols()


def test_host_only_calls(lib):
    lib.mpsgpu_status_string.restype = ctypes.c_char_p
    assert lib.mpsgpu_status_string(0) == b"ok"
    assert lib.mpsgpu_status_string(3) == b"energy increase"
    from mpsdyn_b200 import capi
    o = capi.Options()
    lib.mpsgpu_default_options(ctypes.byref(o))
    assert o.convtol == 1e-5 and o.eigtol == 0.0 and o.max_krylov == 64
