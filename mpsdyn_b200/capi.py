"""ctypes binding of libmpsgpu (include/mpsgpu.h) for tests, benchmarks and
Python callers.  Arrays cross the boundary in the reference layout
(column-major complex128).  There is no CPU fallback: if the library or a
GPU is missing, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpsgpu.so")

STATUS = {
    0: "ok", 1: "bad shape", 2: "not converged", 3: "energy increase", 4: "non-finite value",
    5: "out of memory", 6: "cancelled", 7: "timeout", 8: "CUDA error", 9: "invalid argument",
}

EXPORTS = [
    "mpsgpu_default_options", "mpsgpu_create", "mpsgpu_destroy", "mpsgpu_status_string",
    "mpsgpu_last_error", "mpsgpu_launch_count", "mpsgpu_synchronize", "mpsgpu_get_stream",
    "mpsgpu_profile_begin", "mpsgpu_profile_end", "mpsgpu_profile_kernels", "mpsgpu_mpo_upload",
    "mpsgpu_mpo_free", "mpsgpu_mpo_info", "mpsgpu_mpo_download", "mpsgpu_mpo_ising", "mpsgpu_mpo_ising_evolution", "mpsgpu_mpo_schwinger", "mpsgpu_mpo_heisenberg", "mpsgpu_mpo_bosehubbard",
    "mpsgpu_mps_upload", "mpsgpu_mps_random", "mpsgpu_mps_random_state", "mpsgpu_mps_product",
    "mpsgpu_mps_copy", "mpsgpu_mps_info", "mpsgpu_mps_download", "mpsgpu_mps_free",
    "mpsgpu_mps_export", "mpsgpu_mps_import", "mpsgpu_mpo_save", "mpsgpu_mpo_load",
    "mpsgpu_optimize_sum", "mpsgpu_optimize_mps",
    "mpsgpu_mps_gauge", "mpsgpu_mps_gauge_cond", "mpsgpu_mps_increase_bond", "mpsgpu_mps_bond", "mpsgpu_mps_set_normfact", "mpsgpu_mps_approximate", "mpsgpu_mps_apply_mpo", "mpsgpu_find_ground_state", "mpsgpu_find_ground_state_two_site", "mpsgpu_find_next_excited_state",
    "mpsgpu_find_ground_state_batch", "mpsgpu_find_next_excited_state_batch",
    "mpsgpu_optimize", "mpsgpu_contract", "mpsgpu_contract2", "mpsgpu_expectation_local", "mpsgpu_entropy",
    "mpsgpu_schmidt_values", "mpsgpu_heff_matvec", "mpsgpu_heff_matvec_grouped", "mpsgpu_heff_matvec_grouped_ex", "mpsgpu_zgemm_split", "mpsgpu_set_autotune", "mpsgpu_autotune_entries",
    "mpsgpu_env_left", "mpsgpu_env_right",
    "mpsgpu_qr", "mpsgpu_lq", "mpsgpu_qr_device_noalloc",
    "mpsgpu_server_create", "mpsgpu_server_submit", "mpsgpu_server_poll", "mpsgpu_server_cancel",
    "mpsgpu_server_drain", "mpsgpu_request_footprint", "mpsgpu_server_destroy",
]


# kernel classes of mpsgpu_profile_kernels (work units: flops, BF16 tensor
# flops, bytes, flops); one launch in 32 of each class is sampled
PROFILE_CLASSES = ("gemm_fp64_dmma", "gemm_split_tcgen05", "lanczos_step", "qr", "split_operands")


class Options(C.Structure):
    _fields_ = [
        ("convtol", C.c_double), ("eigtol", C.c_double), ("excorthtol", C.c_double),
        ("max_rounds", C.c_int), ("max_krylov", C.c_int), ("precision", C.c_int),
        ("verbose", C.c_int), ("cancel_flag", C.c_void_p),
        ("checkpoint_file", C.c_char_p), ("checkpoint_every", C.c_int), ("checkpoint_seconds", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("rounds", C.c_int), ("site_solves", C.c_longlong), ("matvecs", C.c_longlong),
        ("env_updates", C.c_longlong), ("qr_calls", C.c_longlong), ("flops", C.c_double),
        ("seconds", C.c_double), ("matvec_seconds", C.c_double),
        ("split_matvecs", C.c_longlong), ("split_rounds", C.c_int),
        ("host_launch_seconds", C.c_double), ("host_wait_seconds", C.c_double),
        ("host_tridiag_seconds", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class MpsgpuError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"mpsgpu: {STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libmpsgpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (run mpsdyn_b200/build.py)")
        lib = C.CDLL(path)
        P = C.c_void_p
        lib.mpsgpu_status_string.restype = C.c_char_p
        lib.mpsgpu_last_error.restype = C.c_char_p
        lib.mpsgpu_last_error.argtypes = [P]
        lib.mpsgpu_launch_count.restype = C.c_longlong
        lib.mpsgpu_launch_count.argtypes = [P]
        lib.mpsgpu_default_options.argtypes = [C.POINTER(Options)]
        lib.mpsgpu_mps_random.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(P)]
        lib.mpsgpu_mps_random_state.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(P)]
        lib.mpsgpu_find_ground_state.argtypes = [P, P, C.c_int, C.c_double, C.POINTER(Options), P,
                                                 C.POINTER(C.c_double), C.POINTER(Stats)]
        lib.mpsgpu_find_ground_state_two_site.argtypes = [P, P, C.c_int, C.c_double, C.POINTER(Options), P,
                                                          C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(Stats)]
        lib.mpsgpu_find_next_excited_state.argtypes = [P, P, C.c_int, C.POINTER(P), C.c_int, C.c_double,
                                                       C.POINTER(Options), P, C.POINTER(C.c_double),
                                                       C.POINTER(Stats)]
        lib.mpsgpu_optimize.argtypes = [P, P, P, P, C.c_int, C.POINTER(Options), C.POINTER(C.c_double),
                                        C.POINTER(C.c_double), C.POINTER(Stats)]
        lib.mpsgpu_mps_upload.argtypes = [P, C.c_int, P, P, C.c_double, C.POINTER(P)]
        lib.mpsgpu_heff_matvec.argtypes = [P, P, P, P, P, P, P, P, P, C.c_double, C.c_int]
        lib.mpsgpu_entropy.argtypes = [P, P, C.c_int, C.POINTER(C.c_double)]
        lib.mpsgpu_mps_gauge.argtypes = [P, P, C.c_char]
        lib.mpsgpu_mps_approximate.argtypes = [P, P, C.c_int, C.POINTER(P), C.POINTER(C.c_double)]
        lib.mpsgpu_mps_apply_mpo.argtypes = [P, P, P, C.c_int, C.c_int, C.c_char, C.POINTER(P),
                                             C.POINTER(C.c_double)]
        D_ = C.c_double
        lib.mpsgpu_mpo_ising.argtypes = [P, C.c_int, D_, D_, D_, C.POINTER(P)]
        lib.mpsgpu_mpo_ising_evolution.argtypes = [P, C.c_int, D_, D_, D_, D_, C.c_int, C.POINTER(P)]
        lib.mpsgpu_mpo_schwinger.argtypes = [P, C.c_int, D_, D_, D_, D_, C.POINTER(P)]
        lib.mpsgpu_mpo_heisenberg.argtypes = [P, C.c_int, D_, D_, D_, D_, D_, D_, D_, C.POINTER(P)]
        lib.mpsgpu_mpo_bosehubbard.argtypes = [P, C.c_int, C.c_int, D_, D_, C.c_int, D_, D_, C.POINTER(P)]
        lib.mpsgpu_mps_import.argtypes = [P, C.c_char_p, C.POINTER(P)]
        lib.mpsgpu_mps_export.argtypes = [P, P, C.c_char_p]
        lib.mpsgpu_mpo_load.argtypes = [P, C.c_char_p, C.POINTER(P)]
        lib.mpsgpu_mpo_save.argtypes = [P, P, C.c_char_p]
        lib.mpsgpu_optimize_sum.argtypes = [P, C.c_int, P, P, P, C.c_int, C.POINTER(Options), C.POINTER(Stats)]
        lib.mpsgpu_optimize_mps.argtypes = [P, P, P, C.c_int, C.POINTER(Options), C.POINTER(C.c_double),
                                            C.POINTER(Stats)]
        _lib = lib
    return _lib


def _fortran(a) -> np.ndarray:
    return np.asfortranarray(np.asarray(a, dtype=np.complex128))


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def _ints(v) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v, dtype=np.int32))


class Context:
    """One CUDA stream on one device, and the objects created on it."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        self._check(self.lib.mpsgpu_create(device, C.byref(h)), ctx=False)
        self.h = h

    def _check(self, st: int, ctx: bool = True) -> None:
        if st != 0:
            msg = self.lib.mpsgpu_last_error(self.h).decode() if ctx else ""
            raise MpsgpuError(st, msg)

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.mpsgpu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def launches(self) -> int:
        return int(self.lib.mpsgpu_launch_count(self.h))

    def synchronize(self) -> None:
        self._check(self.lib.mpsgpu_synchronize(self.h))

    @property
    def stream(self) -> int:
        """The context's cudaStream_t as an integer handle."""
        s = C.c_void_p()
        self._check(self.lib.mpsgpu_get_stream(self.h, C.byref(s)))
        return s.value or 0

    def profile_begin(self) -> None:
        self._check(self.lib.mpsgpu_profile_begin(self.h))

    def profile_end(self) -> dict:
        ms, fl, n = C.c_double(), C.c_double(), C.c_longlong()
        self._check(self.lib.mpsgpu_profile_end(self.h, C.byref(ms), C.byref(fl), C.byref(n)))
        out = {"gemm_ms": ms.value, "gemm_flops": fl.value, "gemm_calls": n.value}
        nc = len(PROFILE_CLASSES)
        kms, kwork, kcalls = (C.c_double * nc)(), (C.c_double * nc)(), (C.c_longlong * nc)()
        self._check(self.lib.mpsgpu_profile_kernels(self.h, kms, kwork, kcalls))
        out["kernels"] = {name: {"ms": kms[i], "work": kwork[i], "calls": kcalls[i]}
                          for i, name in enumerate(PROFILE_CLASSES)}
        return out

    # ---- objects ----
    def mpo(self, ops: list) -> "DeviceMPO":
        arrs = [_fortran(w) for w in ops]
        dims = _ints([s for w in arrs for s in w.shape])
        ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        h = C.c_void_p()
        self._check(self.lib.mpsgpu_mpo_upload(self.h, len(arrs), _ptr(dims), ptrs, C.byref(h)))
        return DeviceMPO(self, h, len(arrs))

    def mpo_ising(self, L: int, J: float, g: float, h: float) -> "DeviceMPO":
        h_ = C.c_void_p()
        self._check(self.lib.mpsgpu_mpo_ising(self.h, L, J, g, h, C.byref(h_)))
        return DeviceMPO(self, h_, L)

    def mpo_ising_evolution(self, L: int, J: float, g: float, h: float, delta: float, imag: bool) -> "DeviceMPO":
        h_ = C.c_void_p()
        self._check(self.lib.mpsgpu_mpo_ising_evolution(self.h, L, J, g, h, delta, int(imag), C.byref(h_)))
        return DeviceMPO(self, h_, L)

    def mpo_schwinger(self, N: int, mu: float, x: float, l0: float = 0.0, alpha: float = 0.0) -> "DeviceMPO":
        h_ = C.c_void_p()
        self._check(self.lib.mpsgpu_mpo_schwinger(self.h, N, mu, x, l0, alpha, C.byref(h_)))
        return DeviceMPO(self, h_, N)

    def mpo_heisenberg(self, L: int, Jx: float, Jy: float, Jz: float, hx: float = 0.0, hy: float = 0.0,
                       hz: float = 0.0, offset: float = 0.0) -> "DeviceMPO":
        h_ = C.c_void_p()
        self._check(self.lib.mpsgpu_mpo_heisenberg(self.h, L, Jx, Jy, Jz, hx, hy, hz, offset, C.byref(h_)))
        return DeviceMPO(self, h_, L)

    def mpo_bosehubbard(self, L: int, N: int, t: float, U: float, Ntarget: int, penN: float,
                        V: float = 0.0) -> "DeviceMPO":
        h_ = C.c_void_p()
        self._check(self.lib.mpsgpu_mpo_bosehubbard(self.h, L, N, t, U, Ntarget, penN, V, C.byref(h_)))
        return DeviceMPO(self, h_, L)

    def mps(self, sites: list, normfact: float = 1.0) -> "DeviceMPS":
        arrs = [_fortran(a) for a in sites]
        dims = _ints([s for a in arrs for s in a.shape])
        ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
        h = C.c_void_p()
        self._check(self.lib.mpsgpu_mps_upload(self.h, len(arrs), _ptr(dims), ptrs, float(normfact), C.byref(h)))
        return DeviceMPS(self, h)

    def mps_random(self, L: int, d: int, D: int, seed: int) -> "DeviceMPS":
        h = C.c_void_p()
        self._check(self.lib.mpsgpu_mps_random(self.h, L, d, D, C.c_uint64(seed), C.byref(h)))
        return DeviceMPS(self, h)

    def mps_random_state(self, L: int, d: int, D: int, seed: int) -> "DeviceMPS":
        """MPS::setRandomState: the random sites right-gauged, norm 1."""
        h = C.c_void_p()
        self._check(self.lib.mpsgpu_mps_random_state(self.h, L, d, D, C.c_uint64(seed), C.byref(h)))
        return DeviceMPS(self, h)

    def mps_product(self, L: int, d: int, D: int) -> "DeviceMPS":
        h = C.c_void_p()
        self._check(self.lib.mpsgpu_mps_product(self.h, L, d, D, C.byref(h)))
        return DeviceMPS(self, h)

    @staticmethod
    def options(convtol=1e-5, eigtol=0.0, excorthtol=0.0, max_rounds=1000, max_krylov=64,
                precision=0, verbose=0, checkpoint_file=None, checkpoint_every=200,
                checkpoint_seconds=0.0) -> Options:
        o = Options(convtol, eigtol, excorthtol, max_rounds, max_krylov, precision, verbose)
        if checkpoint_file:
            o._ckpt = str(checkpoint_file).encode()  # kept alive with the struct
            o.checkpoint_file = o._ckpt
        o.checkpoint_every = checkpoint_every
        o.checkpoint_seconds = checkpoint_seconds
        return o

    # ---- files in the reference's binary formats ----
    def mps_import(self, filename: str) -> "DeviceMPS":
        h = C.c_void_p()
        self._check(self.lib.mpsgpu_mps_import(self.h, str(filename).encode(), C.byref(h)))
        return DeviceMPS(self, h)

    def mps_export(self, mps: "DeviceMPS", filename: str) -> None:
        self._check(self.lib.mpsgpu_mps_export(self.h, mps.h, str(filename).encode()))

    def mpo_load(self, filename: str) -> "DeviceMPO":
        h = C.c_void_p()
        self._check(self.lib.mpsgpu_mpo_load(self.h, str(filename).encode(), C.byref(h)))
        L = C.c_int()
        self._check(self.lib.mpsgpu_mpo_info(self.h, h, C.byref(L), None))
        return DeviceMPO(self, h, L.value)

    def mpo_save(self, mpo: "DeviceMPO", filename: str) -> None:
        self._check(self.lib.mpsgpu_mpo_save(self.h, mpo.h, str(filename).encode()))

    # ---- Contractor ----
    def find_ground_state(self, ops: "DeviceMPO", D: int, init: "DeviceMPS", offset: float = 0.0,
                          opts: Options = None):
        e = C.c_double()
        st = Stats()
        o = opts or self.options()
        self._check(self.lib.mpsgpu_find_ground_state(self.h, ops.h, D, offset, C.byref(o), init.h,
                                                      C.byref(e), C.byref(st)))
        return e.value, st.as_dict()

    def find_ground_state_two_site(self, ops: "DeviceMPO", D: int, init: "DeviceMPS", offset: float = 0.0,
                                   opts: Options = None):
        """Two-site DMRG; returns (energy, max relative discarded weight, stats)."""
        e, dw = C.c_double(), C.c_double()
        st = Stats()
        o = opts or self.options()
        self._check(self.lib.mpsgpu_find_ground_state_two_site(self.h, ops.h, D, offset, C.byref(o), init.h,
                                                               C.byref(e), C.byref(dw), C.byref(st)))
        return e.value, dw.value, st.as_dict()

    def find_next_excited_state(self, ops, D, levels, init, offset=0.0, opts=None):
        e = C.c_double()
        st = Stats()
        o = opts or self.options()
        arr = (C.c_void_p * len(levels))(*[lv.h.value for lv in levels])
        self._check(self.lib.mpsgpu_find_next_excited_state(self.h, ops.h, D, arr, len(levels), offset,
                                                            C.byref(o), init.h, C.byref(e), C.byref(st)))
        return e.value, st.as_dict()

    def find_ground_state_batch(self, ops: list, D: int, inits: list, offset: float = 0.0, opts=None):
        """mpsgpu_find_ground_state_batch: solves swept in lockstep; returns
        (energies, statuses, stats dicts); raises only on a call-level error."""
        n = len(inits)
        P = C.c_void_p
        e = (C.c_double * n)()
        stv = (C.c_int * n)()
        sts = (Stats * n)()
        o = opts or self.options()
        r = self.lib.mpsgpu_find_ground_state_batch(self.h, n, (P * n)(*[m.h for m in ops]), D, C.c_double(offset),
                                                    C.byref(o), (P * n)(*[s.h for s in inits]), e, stv, sts)
        if r != 0 and all(v == 0 for v in stv):
            self._check(r)
        return list(e), list(stv), [x.as_dict() for x in sts]

    def find_next_excited_state_batch(self, ops: list, D: int, levels: list, inits: list, offset: float = 0.0,
                                      opts=None):
        """levels[i]: the list of states solve i projects out."""
        n = len(inits)
        P = C.c_void_p
        flat = [lv.h for group in levels for lv in group]
        e = (C.c_double * n)()
        stv = (C.c_int * n)()
        sts = (Stats * n)()
        o = opts or self.options()
        r = self.lib.mpsgpu_find_next_excited_state_batch(
            self.h, n, (P * n)(*[m.h for m in ops]), D, (P * len(flat))(*flat),
            (C.c_int * n)(*[len(g) for g in levels]), C.c_double(offset), C.byref(o),
            (P * n)(*[s.h for s in inits]), e, stv, sts)
        if r != 0 and all(v == 0 for v in stv):
            self._check(r)
        return list(e), list(stv), [x.as_dict() for x in sts]

    def optimize(self, ops, orig, init, D=0, opts=None, want_err=False):
        st = Stats()
        o = opts or self.options()
        en, et = C.c_double(), C.c_double()
        self._check(self.lib.mpsgpu_optimize(self.h, ops.h, orig.h, init.h, D, C.byref(o),
                                             C.byref(en) if want_err else None,
                                             C.byref(et) if want_err else None, C.byref(st)))
        return (en.value, et.value, st.as_dict()) if want_err else st.as_dict()

    def optimize_sum(self, kets: list, beta: list, init: "DeviceMPS", D: int = 0, opts: Options = None) -> dict:
        n = len(kets)
        arr = (C.c_void_p * n)(*[k.h for k in kets])
        b = np.array([[complex(x).real, complex(x).imag] for x in beta], dtype=np.float64).ravel()
        st = Stats()
        o = opts or self.options()
        self._check(self.lib.mpsgpu_optimize_sum(self.h, n, arr, _ptr(b), init.h, D, C.byref(o), C.byref(st)))
        return st.as_dict()

    def optimize_mps(self, ket: "DeviceMPS", init: "DeviceMPS", D: int = 0, opts: Options = None):
        err = C.c_double()
        st = Stats()
        o = opts or self.options()
        self._check(self.lib.mpsgpu_optimize_mps(self.h, ket.h, init.h, D, C.byref(o), C.byref(err), C.byref(st)))
        return err.value, st.as_dict()

    def contract(self, ket, ops, bra) -> complex:
        re, im = C.c_double(), C.c_double()
        self._check(self.lib.mpsgpu_contract(self.h, ket.h, ops.h if ops is not None else None, bra.h,
                                             C.byref(re), C.byref(im)))
        return complex(re.value, im.value)

    def contract2(self, ops, ket, bra=None) -> complex:
        """<bra|ops^dag ops|ket> (bra defaults to ket)."""
        re, im = C.c_double(), C.c_double()
        self._check(self.lib.mpsgpu_contract2(self.h, ops.h, ket.h, bra.h if bra is not None else None,
                                              C.byref(re), C.byref(im)))
        return complex(re.value, im.value)

    def expectation_local(self, mps, op2) -> np.ndarray:
        op = _fortran(op2)
        L = mps.info()[0]
        out = np.zeros(L)
        self._check(self.lib.mpsgpu_expectation_local(self.h, mps.h, _ptr(op), _ptr(out)))
        return out

    def entropy(self, mps, pos: int) -> float:
        s = C.c_double()
        self._check(self.lib.mpsgpu_entropy(self.h, mps.h, pos, C.byref(s)))
        return s.value

    def schmidt_values(self, mps, pos: int) -> np.ndarray:
        cap = 4096
        out = np.zeros(cap)
        n = C.c_int()
        self._check(self.lib.mpsgpu_schmidt_values(self.h, mps.h, pos, _ptr(out), cap, C.byref(n)))
        return out[: n.value].copy()

    # ---- kernel-level ----
    def heff_matvec(self, L, W, R, x, offset=0.0, hermitian=False) -> np.ndarray:
        L, W, R, x = _fortran(L), _fortran(W), _fortran(R), _fortran(x)
        y = np.zeros(W.shape[0] * L.shape[0] * R.shape[0], dtype=np.complex128)
        ld, wd, rd = _ints(L.shape), _ints(W.shape), _ints(R.shape)  # kept alive across the call
        self._check(self.lib.mpsgpu_heff_matvec(
            self.h, _ptr(ld), _ptr(L), _ptr(wd), _ptr(W), _ptr(rd),
            _ptr(R), _ptr(x), _ptr(y), float(offset), int(hermitian)))
        return y

    def env_left(self, T, ket, W, bra) -> np.ndarray:
        T, ket, W, bra = _fortran(T), _fortran(ket), _fortran(W), _fortran(bra)
        out = np.zeros((bra.shape[2], W.shape[3], ket.shape[2]), dtype=np.complex128, order="F")
        td, kd, wd, bd = _ints(T.shape), _ints(ket.shape), _ints(W.shape), _ints(bra.shape)
        self._check(self.lib.mpsgpu_env_left(self.h, _ptr(td), _ptr(T), _ptr(kd), _ptr(ket), _ptr(wd),
                                             _ptr(W), _ptr(bd), _ptr(bra), _ptr(out)))
        return out

    def env_right(self, T, ket, W, bra) -> np.ndarray:
        T, ket, W, bra = _fortran(T), _fortran(ket), _fortran(W), _fortran(bra)
        out = np.zeros((bra.shape[1], W.shape[1], ket.shape[1]), dtype=np.complex128, order="F")
        td, kd, wd, bd = _ints(T.shape), _ints(ket.shape), _ints(W.shape), _ints(bra.shape)
        self._check(self.lib.mpsgpu_env_right(self.h, _ptr(td), _ptr(T), _ptr(kd), _ptr(ket), _ptr(wd),
                                              _ptr(W), _ptr(bd), _ptr(bra), _ptr(out)))
        return out

    def qr(self, A):
        A = _fortran(A)
        m, n = A.shape
        K = min(m, n)
        Q = np.zeros((m, K), dtype=np.complex128, order="F")
        R = np.zeros((K, n), dtype=np.complex128, order="F")
        self._check(self.lib.mpsgpu_qr(self.h, m, n, _ptr(A), _ptr(Q), _ptr(R)))
        return Q, R

    def lq(self, A):
        A = _fortran(A)
        m, n = A.shape
        K = min(m, n)
        Lm = np.zeros((m, K), dtype=np.complex128, order="F")
        Q = np.zeros((K, n), dtype=np.complex128, order="F")
        self._check(self.lib.mpsgpu_lq(self.h, m, n, _ptr(A), _ptr(Lm), _ptr(Q)))
        return Lm, Q


class DeviceMPO:
    def __init__(self, ctx: Context, h, L: int):
        self.ctx, self.h, self.L = ctx, h, L

    def download(self) -> list:
        """The operator tensors W(du, Dl, dd, Dr) back on the host."""
        L = C.c_int()
        self.ctx._check(self.ctx.lib.mpsgpu_mpo_info(self.ctx.h, self.h, C.byref(L), None))
        dims = np.zeros(4 * L.value, dtype=np.int32)
        self.ctx._check(self.ctx.lib.mpsgpu_mpo_info(self.ctx.h, self.h, C.byref(L), _ptr(dims)))
        ws = [np.zeros(tuple(d), dtype=np.complex128, order="F") for d in dims.reshape(L.value, 4)]
        ptrs = (C.c_void_p * L.value)(*[w.ctypes.data for w in ws])
        self.ctx._check(self.ctx.lib.mpsgpu_mpo_download(self.ctx.h, self.h, ptrs))
        return ws

    def free(self) -> None:
        if self.h:
            self.ctx.lib.mpsgpu_mpo_free(self.ctx.h, self.h)
            self.h = None


class DeviceMPS:
    def __init__(self, ctx: Context, h):
        self.ctx, self.h = ctx, h

    def info(self):
        L = C.c_int()
        self.ctx._check(self.ctx.lib.mpsgpu_mps_info(self.ctx.h, self.h, C.byref(L), None, None))
        dims = np.zeros(3 * L.value, dtype=np.int32)
        nf = C.c_double()
        self.ctx._check(self.ctx.lib.mpsgpu_mps_info(self.ctx.h, self.h, C.byref(L), _ptr(dims), C.byref(nf)))
        return L.value, dims.reshape(L.value, 3), nf.value

    def download(self):
        L, dims, nf = self.info()
        sites = [np.zeros(tuple(d), dtype=np.complex128, order="F") for d in dims]
        ptrs = (C.c_void_p * L)(*[a.ctypes.data for a in sites])
        self.ctx._check(self.ctx.lib.mpsgpu_mps_download(self.ctx.h, self.h, ptrs))
        return sites, nf

    def copy(self) -> "DeviceMPS":
        h = C.c_void_p()
        self.ctx._check(self.ctx.lib.mpsgpu_mps_copy(self.ctx.h, self.h, C.byref(h)))
        return DeviceMPS(self.ctx, h)

    def gauge(self, direction: str) -> None:
        self.ctx._check(self.ctx.lib.mpsgpu_mps_gauge(self.ctx.h, self.h, direction.encode()))

    def approximate(self, D: int):
        """MPS(self, D): a copy cut to bond D; returns (DeviceMPS, discarded weight)."""
        h, disc = C.c_void_p(), C.c_double()
        self.ctx._check(self.ctx.lib.mpsgpu_mps_approximate(self.ctx.h, self.h, D, C.byref(h), C.byref(disc)))
        return DeviceMPS(self.ctx, h), disc.value

    def apply_mpo(self, ops: "DeviceMPO", D: int = 0, dagger: bool = False, direction: str = "L"):
        """ops|self> applied exactly (D <= 0) or cut to D (MPS::truncate);
        returns (DeviceMPS, discarded weight)."""
        h, disc = C.c_void_p(), C.c_double()
        self.ctx._check(self.ctx.lib.mpsgpu_mps_apply_mpo(self.ctx.h, ops.h, self.h, D, int(dagger),
                                                          direction.encode(), C.byref(h), C.byref(disc)))
        return DeviceMPS(self.ctx, h), disc.value

    def free(self) -> None:
        if self.h:
            self.ctx.lib.mpsgpu_mps_free(self.ctx.h, self.h)
            self.h = None


def qr_device_noalloc(m: int, n: int, a_ptr: int, q_ptr: int, r_ptr: int, stream: int = 0) -> None:
    """mpsgpu_qr_device_noalloc on device pointers (integers): QR of the m x n
    column-major complex128 matrix at a_ptr into Q (m x K) and R (K x n)
    without any allocation; asynchronous on `stream`."""
    lib = load()
    P = C.c_void_p
    lib.mpsgpu_qr_device_noalloc.argtypes = [C.c_int, C.c_int, P, P, P, P]
    st = lib.mpsgpu_qr_device_noalloc(m, n, P(a_ptr), P(q_ptr or None), P(r_ptr or None), P(stream or None))
    if st != 0:
        raise MpsgpuError(st, "mpsgpu_qr_device_noalloc")


class HeffInstance(C.Structure):
    _fields_ = [("d", C.c_int), ("wl", C.c_int), ("wr", C.c_int), ("Dl", C.c_int), ("Dr", C.c_int),
                ("L", C.c_void_p), ("W", C.c_void_p), ("Rt", C.c_void_p), ("x", C.c_void_p), ("y", C.c_void_p)]


def heff_matvec_grouped(ctx: "Context", instances: list, repeats: int = 0):
    """mpsgpu_heff_matvec_grouped.  `instances`: dicts with d, wl, wr, Dl, Dr and
    device pointers (integers) L, W, Rt, x, y in the library's layouts.
    Returns (ms_per_run or None, flops per grouped product)."""
    lib = ctx.lib
    P = C.c_void_p
    lib.mpsgpu_heff_matvec_grouped.argtypes = [P, C.c_int, C.POINTER(HeffInstance), C.c_int,
                                               C.POINTER(C.c_double), C.POINTER(C.c_double)]
    arr = (HeffInstance * len(instances))()
    for i, s in enumerate(instances):
        arr[i] = HeffInstance(s["d"], s["wl"], s["wr"], s["Dl"], s["Dr"], s["L"], s["W"], s["Rt"], s["x"], s["y"])
    ms, fl = C.c_double(), C.c_double()
    ctx._check(lib.mpsgpu_heff_matvec_grouped(ctx.h, len(instances), arr, repeats, C.byref(ms), C.byref(fl)))
    return (ms.value if repeats > 0 else None), fl.value


def heff_matvec_grouped_ex(ctx: "Context", instances: list, precision: int = 0, repeats: int = 0):
    """mpsgpu_heff_matvec_grouped_ex: as heff_matvec_grouped with a precision
    choice (0 FP64, 1 split).  Returns (ms_per_run or None, flops, ms_prepare)."""
    lib = ctx.lib
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    lib.mpsgpu_heff_matvec_grouped_ex.argtypes = [P, C.c_int, C.POINTER(HeffInstance), C.c_int, C.c_int, D, D, D]
    arr = (HeffInstance * len(instances))()
    for i, s in enumerate(instances):
        arr[i] = HeffInstance(s["d"], s["wl"], s["wr"], s["Dl"], s["Dr"], s["L"], s["W"], s["Rt"], s["x"], s["y"])
    ms, fl, mp = C.c_double(), C.c_double(), C.c_double()
    ctx._check(lib.mpsgpu_heff_matvec_grouped_ex(ctx.h, len(instances), arr, precision, repeats, C.byref(ms),
                                                 C.byref(fl), C.byref(mp)))
    return (ms.value if repeats > 0 else None), fl.value, mp.value


def set_autotune(on: bool) -> None:
    """mpsgpu_set_autotune: the FP64 GEMM autotuner on or off (process-wide)."""
    lib = load()
    lib.mpsgpu_set_autotune.argtypes = [C.c_int]
    lib.mpsgpu_set_autotune(1 if on else 0)


def autotune_entries() -> int:
    lib = load()
    lib.mpsgpu_autotune_entries.restype = C.c_longlong
    return int(lib.mpsgpu_autotune_entries())


def zgemm_split(ctx: "Context", A: np.ndarray, B: np.ndarray, repeats: int = 0):
    """mpsgpu_zgemm_split: A @ B (complex) in split precision on the tensor
    cores.  Returns (C, ms_total or None, ms_mma or None)."""
    lib = ctx.lib
    P = C.c_void_p
    D = C.POINTER(C.c_double)
    lib.mpsgpu_zgemm_split.argtypes = [P, C.c_int, C.c_int, C.c_int, D, C.c_int, D, C.c_int, D, C.c_int,
                                       C.c_int, D, D]
    A = np.asfortranarray(A, dtype=np.complex128)
    B = np.asfortranarray(B, dtype=np.complex128)
    m, k = A.shape
    k2, n = B.shape
    if k != k2:
        raise ValueError("inner dimensions differ")
    out = np.zeros((m, n), dtype=np.complex128, order="F")
    dp = lambda a: a.ctypes.data_as(D)
    t1, t2 = C.c_double(), C.c_double()
    ctx._check(lib.mpsgpu_zgemm_split(ctx.h, m, n, k, dp(A), m, dp(B), k, dp(out), m, repeats,
                                      C.byref(t1), C.byref(t2)))
    return out, (t1.value if repeats > 0 else None), (t2.value if repeats > 0 else None)


class Request(C.Structure):
    _fields_ = [("model", C.c_int), ("L", C.c_int), ("D", C.c_int), ("p0", C.c_double), ("p1", C.c_double),
                ("p2", C.c_double), ("seed", C.c_uint64), ("convtol", C.c_double), ("precision", C.c_int),
                ("kind", C.c_int), ("steps", C.c_int), ("dt", C.c_double), ("imag", C.c_int),
                ("obs_sx", C.c_void_p), ("obs_entropy", C.c_void_p), ("result_file", C.c_char_p)]


KIND_GROUND_STATE, KIND_TIME_EVOLUTION = 0, 1


class Result(C.Structure):
    _fields_ = [("id", C.c_uint64), ("status", C.c_int), ("energy", C.c_double), ("rounds", C.c_int),
                ("matvecs", C.c_longlong), ("flops", C.c_double), ("t_submit", C.c_double),
                ("t_start", C.c_double), ("t_end", C.c_double), ("footprint_bytes", C.c_longlong)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


MODEL_ISING, MODEL_SCHWINGER = 0, 1


class Server:
    """mpsgpu_server: continuous batching of ground-state requests on one GPU."""

    def __init__(self, device: int = 0, slots: int = 8, hbm_budget_bytes: int = 64 << 30):
        self.lib = load()
        P = C.c_void_p
        self.lib.mpsgpu_server_create.argtypes = [C.c_int, C.c_int, C.c_longlong, C.POINTER(P)]
        self.lib.mpsgpu_server_submit.argtypes = [P, C.POINTER(Request), C.POINTER(C.c_uint64)]
        self.lib.mpsgpu_server_poll.argtypes = [P, C.POINTER(Result), C.c_int, C.POINTER(C.c_int)]
        self.lib.mpsgpu_server_cancel.argtypes = [P, C.c_uint64]
        self.lib.mpsgpu_server_drain.argtypes = [P, C.c_double]
        self.lib.mpsgpu_server_destroy.argtypes = [P]
        self.lib.mpsgpu_request_footprint.argtypes = [C.POINTER(Request)]
        self.lib.mpsgpu_request_footprint.restype = C.c_longlong
        self._keep = []
        h = P()
        st = self.lib.mpsgpu_server_create(device, slots, hbm_budget_bytes, C.byref(h))
        if st != 0:
            raise MpsgpuError(st, "mpsgpu_server_create")
        self.h = h

    def submit(self, model: int, L: int, D: int, p0: float, p1: float, p2: float, seed: int,
               convtol: float = 1e-10, precision: int = 0, result_file: str = None) -> int:
        """A ground-state request (mpsgpu_request, kind 0)."""
        r = Request(model, L, D, p0, p1, p2, seed, convtol, precision)
        return self._submit(r, result_file)

    def submit_evolution(self, L: int, D: int, J: float, g: float, h: float, steps: int, dt: float,
                         imag: bool = False, convtol: float = 1e-10, observe: bool = True,
                         result_file: str = None) -> tuple:
        """A time-evolution request (kind 1) of the open Ising chain from
        |0...0>; returns (id, sx, entropy): arrays (length steps) the server
        fills with <sigma_x> at site L/2 and the entropy of bond L/2 after
        every step."""
        r = Request(MODEL_ISING, L, D, J, g, h, 0, convtol, 0)
        r.kind = KIND_TIME_EVOLUTION
        r.steps, r.dt, r.imag = steps, dt, int(bool(imag))
        sx = np.full(steps, np.nan)
        ent = np.full(steps, np.nan)
        if observe:
            r.obs_sx, r.obs_entropy = sx.ctypes.data, ent.ctypes.data
            self._keep.append((sx, ent))  # the server writes into them until the result is polled
        return self._submit(r, result_file), sx, ent

    def _submit(self, r: Request, result_file) -> int:
        if result_file:
            r.result_file = str(result_file).encode()
        rid = C.c_uint64()
        st = self.lib.mpsgpu_server_submit(self.h, C.byref(r), C.byref(rid))
        if st != 0:
            raise MpsgpuError(st, "mpsgpu_server_submit")
        return rid.value

    def footprint(self, model: int, L: int, D: int, precision: int = 0, kind: int = 0) -> int:
        r = Request(model, L, D, 0, 0, 0, 0, 0, precision)
        r.kind = kind
        return int(self.lib.mpsgpu_request_footprint(C.byref(r)))

    def poll(self) -> list:
        buf = (Result * 256)()
        n = C.c_int()
        out = []
        while True:
            st = self.lib.mpsgpu_server_poll(self.h, buf, 256, C.byref(n))
            if st != 0:
                raise MpsgpuError(st, "mpsgpu_server_poll")
            out.extend(buf[i].as_dict() for i in range(n.value))
            if n.value < 256:
                return out

    def cancel(self, rid: int) -> None:
        st = self.lib.mpsgpu_server_cancel(self.h, rid)
        if st != 0:
            raise MpsgpuError(st, "mpsgpu_server_cancel")

    def drain(self, timeout_s: float = 0.0) -> bool:
        return self.lib.mpsgpu_server_drain(self.h, timeout_s) == 0

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.mpsgpu_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
