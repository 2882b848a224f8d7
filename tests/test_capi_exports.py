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


def test_request_footprint_counts_split_buffers(lib):
    """Admission by HBM footprint (host arithmetic only): a split-precision
    request reserves, on top of the FP64 one, the BF16 limb planes of L, Rt,
    x and T2 and the FP64 intermediates of the split products (T1 in up to 4
    K chunks, T2, the last product in up to 8 K chunks), for ground states and
    time evolutions alike."""
    from mpsdyn_b200 import capi
    lib.mpsgpu_request_footprint.argtypes = [ctypes.POINTER(capi.Request)]
    lib.mpsgpu_request_footprint.restype = ctypes.c_longlong

    def fp(kind, precision, D, L=64):
        r = capi.Request(0, L, D, 0, 0, 0, 0, 0, precision)
        r.kind = kind
        return lib.mpsgpu_request_footprint(ctypes.byref(r))

    def planes(rows, K):
        return 12 * ((rows + 127) // 128 * 128) * ((K + 15) // 16 * 16)

    for kind, w in ((capi.KIND_GROUND_STATE, 3), (capi.KIND_TIME_EVOLUTION, 2)):
        for D in (32, 128, 256):
            d = 2
            extra = (planes(D * w, D) + planes(D, D * w) + planes(d * D, D) + planes(D * d, D * w) +
                     16 * (4 * D * w * d * D + D * d * D * w + 8 * D * d * D))
            assert fp(kind, 1, D) - fp(kind, 0, D) == extra
