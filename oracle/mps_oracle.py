"""CPU restatement of the mpsdyn DMRG hot path -- TEST INFRASTRUCTURE ONLY.

This module is the checker for the CUDA path: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The product library never calls it.

Every function restates one reference function of mcbapo/mpsdyn (paths are
relative to the reference's ``src/``) in numpy.  Tensor conventions follow
the reference exactly:

* site tensor  ``A[s, l, r]``        shape (d, Dl, Dr)        (core/cpp/Site.cpp:16-21)
* MPO tensor   ``W[s', bl, s, br]``  shape (du, Dl, dd, Dr)   (core/cpp/Operator.cpp:17-24)
* environments ``L[bra, w, ket]`` and ``R[bra, w, ket]``     (core/cpp/Operator.cpp:273-387)
* local vector ``x = vec_F(A)`` (column-major, s fastest)     (wrapper/multipliers/TensorMultiplier.h:28)

Parity of this restatement is pinned against the reference itself, compiled
from source into ``oracle/_ref`` (``oracle/Makefile``), through the golden
fixtures in ``tests/golden`` written by ``tests/golden/make_golden.py``.
"""
from __future__ import annotations

import math
import struct
from dataclasses import dataclass, field

import numpy as np

# ---------------------------------------------------------------------------
# Binary formats (wrapper/mwArray.cpp:382-442, core/cpp/MPS.cpp:442-509,
# core/cpp/Site.cpp:561-578)
# ---------------------------------------------------------------------------


def write_mwarray(f, arr: np.ndarray) -> None:
    """mwArray::save: int rank, int dims[rank], double[2n] column-major re/im."""
    arr = np.asarray(arr, dtype=np.complex128)
    f.write(struct.pack("<i", arr.ndim))
    f.write(struct.pack("<%di" % arr.ndim, *arr.shape))
    f.write(np.asfortranarray(arr).ravel(order="F").view(np.float64).tobytes())


def read_mwarray(f) -> np.ndarray:
    """mwArray::load."""
    (rank,) = struct.unpack("<i", f.read(4))
    dims = struct.unpack("<%di" % rank, f.read(4 * rank))
    n = int(np.prod(dims)) if rank else 1
    data = np.frombuffer(f.read(16 * n), dtype=np.float64).copy().view(np.complex128)
    return data.reshape(dims, order="F")


def save_array(fn: str, arr: np.ndarray) -> None:
    with open(fn, "wb") as f:
        write_mwarray(f, arr)


def load_array(fn: str) -> np.ndarray:
    with open(fn, "rb") as f:
        return read_mwarray(f)


@dataclass
class MPS:
    """State as the reference keeps it: site tensors, norm factor, gauge tag."""

    sites: list
    normfact: float = 1.0
    gauge: int = 0  # enum Gauge (core/headers/MPS.h:50): gNone=0
    bond: int = 0

    @property
    def L(self) -> int:
        return len(self.sites)

    def copy(self) -> "MPS":
        return MPS([a.copy() for a in self.sites], self.normfact, self.gauge, self.bond)

    def max_bond(self) -> int:
        return max(max(a.shape[1], a.shape[2]) for a in self.sites)


def write_mps(fn: str, mps: MPS) -> None:
    """MPS::exportMPS: int length, int bond, double normfact, int gauge, then
    per site int pos + mwArray (positions 1-based as Site stores them)."""
    bond = mps.bond or mps.max_bond()
    with open(fn, "wb") as f:
        f.write(struct.pack("<iidi", mps.L, bond, mps.normfact, mps.gauge))
        for k, a in enumerate(mps.sites):
            f.write(struct.pack("<i", k + 1))
            write_mwarray(f, a)


def read_mps(fn: str) -> MPS:
    """MPS::importMPS."""
    with open(fn, "rb") as f:
        L, bond, normfact, gauge = struct.unpack("<iidi", f.read(20))
        sites = []
        for _ in range(L):
            f.read(4)
            sites.append(read_mwarray(f))
    return MPS(sites, normfact, gauge, bond)


# ---------------------------------------------------------------------------
# Seeded inputs (this repository's generator, identical in the C-ABI library)
# ---------------------------------------------------------------------------

_M64 = (1 << 64) - 1


def splitmix64(seed: int, counters: np.ndarray) -> np.ndarray:
    """SplitMix64 (Steele, Lea, Flood 2014) evaluated at ``counters``:
    z = seed + (i+1)*0x9E3779B97F4A7C15; z ^= z>>30; z *= 0xBF58476D1CE4E5B9;
    z ^= z>>27; z *= 0x94D049BB133111EB; z ^= z>>31 (all mod 2^64)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed & _M64) + (counters.astype(np.uint64) + np.uint64(1)) * np.uint64(
            0x9E3779B97F4A7C15
        )
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def gaussian_complex(seed: int, offset: int, n: int) -> np.ndarray:
    """n complex N(0,1)-per-component numbers: entry i uses draws 2(offset+i)
    and 2(offset+i)+1 -> uniforms u=((z>>11)+0.5)/2^53 -> Box-Muller
    (re, im) = sqrt(-2 ln u1) (cos 2 pi u2, sin 2 pi u2)."""
    idx = np.arange(2 * offset, 2 * (offset + n), dtype=np.uint64)
    z = splitmix64(seed, idx)
    u = ((z >> np.uint64(11)).astype(np.float64) + 0.5) * (2.0 ** -53)
    u1, u2 = u[0::2], u[1::2]
    r = np.sqrt(-2.0 * np.log(u1))
    return r * np.cos(2 * np.pi * u2) + 1j * r * np.sin(2 * np.pi * u2)


def bond_schedule(L: int, d: int, D: int) -> list:
    """Bond dimensions D_k = min(d^k, d^(L-k), D), k = 0..L (D_0 = D_L = 1):
    what MPS(L,D,d) reaches after gaugeCond('R',1) then gaugeCond('L',1)
    (core/cpp/MPS.cpp:15-35 dims, Site::gaugeR/gaugeL keep K=min(M,N),
    wrapper/qr.cpp:100-102,175-177)."""
    out = []
    for k in range(L + 1):
        out.append(int(min(d ** min(k, 60), d ** min(L - k, 60), D)))
    return out


def random_mps(L: int, d: int, D: int, seed: int) -> MPS:
    """Seeded i.i.d. complex Gaussian MPS on the bond schedule above; entries
    are drawn site by site in column-major order from one counter stream."""
    bonds = bond_schedule(L, d, D)
    sites = []
    off = 0
    for k in range(L):
        shape = (d, bonds[k], bonds[k + 1])
        n = int(np.prod(shape))
        sites.append(gaussian_complex(seed, off, n).reshape(shape, order="F"))
        off += n
    return MPS(sites, 1.0, 0, max(bonds))


def random_state(L: int, d: int, D: int, seed: int) -> MPS:
    """MPS::setRandomState (core/cpp/MPS.cpp:282-294) on the sites of
    random_mps: each site right-gauged in turn, the R factor passed on only
    where the bond shrinks (Site::gaugeR + reduceDimR)."""
    m = random_mps(L, d, D, seed)
    for k in range(L):
        old = m.sites[k].shape
        m.sites[k], tmp = site_gauge_r(m.sites[k])
        if k < L - 1 and m.sites[k].shape[2] != old[2]:
            m.sites[k + 1] = site_reduce_r(m.sites[k + 1], tmp)
    m.gauge = 2
    return m


def product_mps(L: int, d: int, D: int) -> MPS:
    """MPS(L,D,d) of the reference: dims (d,1,D),(d,D,D)...,(d,D,1), each site
    with element (0,0,0)=1 (core/cpp/MPS.cpp:15-35, core/cpp/Site.cpp:16-21)."""
    sites = []
    for k in range(L):
        dl = 1 if k == 0 else D
        dr = 1 if k == L - 1 else D
        a = np.zeros((d, dl, dr), dtype=np.complex128)
        a[0, 0, 0] = 1.0
        sites.append(a)
    return MPS(sites, 1.0, 0, D)


# ---------------------------------------------------------------------------
# MPO builders (models/cpp/IsingHamiltonian.cpp, SchwingerHamiltonian.cpp)
# ---------------------------------------------------------------------------

SIG0 = np.eye(2, dtype=np.complex128)
SIGX = np.array([[0, 1], [1, 0]], dtype=np.complex128)
SIGY = np.array([[0, -1j], [1j, 0]], dtype=np.complex128)
# The reference's Schwinger builder fills its "sigma_y" column-major from
# {0, -i, i, 0} (SchwingerHamiltonian.cpp:30-31), i.e. [[0, i], [-i, 0]].
SIGY_SCHW = np.array([[0, 1j], [-1j, 0]], dtype=np.complex128)
SIGZ = np.array([[1, 0], [0, -1]], dtype=np.complex128)


def _w_from_coeffs(C: np.ndarray, Z: np.ndarray) -> np.ndarray:
    """res = C(Dl*Dr,n) * Z(n,d*d) -> (Dl,Dr,d,d) -> permute(3,1,4,2)
    (IsingHamiltonian.cpp:111-116, SchwingerHamiltonian.cpp:114-118)."""
    Dl, Dr, n = C.shape
    d = Z.shape[1]
    res = C.reshape(Dl * Dr, n, order="F") @ Z.reshape(n, d * d, order="F")
    # Z is (n, d, d) with Z[op, i1, i2] = sigma_op[i1, i2]
    res = res.reshape(Dl, Dr, d, d, order="F")
    return np.ascontiguousarray(res.transpose(2, 0, 3, 1))


def ising_hmpo(L: int, J: float, g: float, h: float, K: float = 0.0) -> list:
    """IsingHamiltonian::setHMPO (IsingHamiltonian.cpp:70-121):
    H = J sum sz sz + g sum sx + h sum sz (+ K offset), MPO bond 3."""
    Z = np.zeros((3, 2, 2), dtype=np.complex128)
    Z[0], Z[1], Z[2] = SIG0, SIGZ, SIGX
    D = 3
    ops = []
    for k in range(L):
        if 1 < k < L - 1:
            ops.append(ops[k - 1])
            continue
        Dl = 1 if k == 0 else D
        Dr = 1 if k == L - 1 else D
        C = np.zeros((Dl, Dr, 3), dtype=np.complex128)
        effJ = 1j * math.sqrt(abs(J)) if J < 0 else math.sqrt(J)
        if k != L - 1:
            C[0, 0, 0] = 1.0
        if k != 0:
            C[Dl - 1, Dr - 1, 0] = 1.0
        C[0, Dr - 1, 2] = g
        C[0, Dr - 1, 1] = h
        C[0, Dr - 1, 0] = K / L
        if k != L - 1:
            C[0, 1, 1] = effJ
        if k != 0:
            C[1, Dr - 1, 1] = effJ
        ops.append(_w_from_coeffs(C, Z))
    return ops


def heisenberg_hmpo(L: int, Jx: float, Jy: float, Jz: float, hx: float = 0.0, hy: float = 0.0,
                    hz: float = 0.0, offset: float = 0.0) -> list:
    """HeisenbergHamiltonian::initHMPO (HeisenbergHamiltonian.cpp:266-331)
    for uniform couplings, d = 2, no Sz penalty: H = sum_k (Jx Sx Sx + Jy Sy Sy
    + Jz Sz Sz)_(k,k+1) + sum_k (hx Sx + hy Sy + hz Sz)_k + offset, spin-1/2
    operators S = sigma / 2; MPO bond 5."""
    Z = np.zeros((4, 2, 2), dtype=np.complex128)
    Z[0], Z[1], Z[2], Z[3] = SIG0, 0.5 * SIGX, 0.5 * SIGY, 0.5 * SIGZ
    D = 5
    ops = []
    for k in range(L):
        Dl = 1 if k == 0 else D
        Dr = 1 if k == L - 1 else D
        C = np.zeros((Dl, Dr, 4), dtype=np.complex128)
        if k != L - 1:
            C[0, 0, 0] = 1.0
            C[0, 1, 1], C[0, 2, 2], C[0, 3, 3] = Jx, Jy, Jz
        if k != 0:
            C[Dl - 1, Dr - 1, 0] = 1.0
            C[1, Dr - 1, 1] = C[2, Dr - 1, 2] = C[3, Dr - 1, 3] = 1.0
        C[0, Dr - 1, 3] = hz
        if hx != 0:
            C[0, Dr - 1, 1] = hx
        if hy != 0:
            C[0, Dr - 1, 2] = hy
        if offset != 0:
            C[0, Dr - 1, 0] = offset / L
        ops.append(_w_from_coeffs(C, Z))
    return ops


def bosehubbard_hmpo(L: int, N: int, t: float, U: float, Ntarget: int, penN: float, V: float = 0.0) -> list:
    """BoseHubbardHamiltonian(L, N, t, U, Ntarget, penN, V) with initZ / initHMPO
    (models/cpp/BoseHubbardHamiltonian.cpp:7-17, 73-160): occupations 0..N
    (d = N + 1), H = -t sum (b+_k b_k+1 + h.c.) + U/2 sum n_k (n_k - 1)
    + V sum n_k + penN (sum n_k - Ntarget)^2, MPO bond 5; the hop is split as
    i sqrt(t) on either side (uniform-coupling form, t >= 0)."""
    if t < 0:
        raise ValueError("bosehubbard_hmpo: t < 0")
    d = N + 1
    Z = np.zeros((6, d, d), dtype=np.complex128)
    for i in range(d):
        Z[0, i, i] = 1.0
        Z[1, i, i] = i * (i - 1)
        if i > 0:
            Z[2, i, i - 1] = math.sqrt(i)      # b+
        if i < N:
            Z[3, i, i + 1] = math.sqrt(i + 1)  # b
        Z[4, i, i] = i
        Z[5, i, i] = i * i
    half_u = 0.5 * U
    hop = 1j * math.sqrt(t)
    D = 5
    ops = []
    for k in range(L):
        Dl = 1 if k == 0 else D
        Dr = 1 if k == L - 1 else D
        C = np.zeros((Dl, Dr, 6), dtype=np.complex128)
        if k != L - 1:
            C[0, 0, 0] = 1.0
            C[0, 1, 2] = hop
            C[0, 2, 3] = hop
            C[0, 3, 4] = 2 * penN
        if k != 0 and k != L - 1:
            C[3, 3, 0] = 1.0
        C[0, Dr - 1, 1] = half_u
        C[0, Dr - 1, 4] = V - 2 * Ntarget * penN
        C[0, Dr - 1, 5] = penN
        C[0, Dr - 1, 0] = penN * Ntarget * Ntarget / L
        if k != 0:
            C[1, Dr - 1, 3] = hop
            C[2, Dr - 1, 2] = hop
            C[3, Dr - 1, 4] = 1.0
            C[Dl - 1, Dr - 1, 0] = 1.0
        ops.append(_w_from_coeffs(C, Z))
    return ops


def _ising_u1(eps: complex, g: float, h: float) -> np.ndarray:
    """isingU1MPO (IsingHamiltonian.cpp:203-218): exp(eps (g sx + h sz))."""
    norm = math.sqrt(g * g + h * h)
    res = np.cosh(norm * eps) * SIG0
    if norm != 0:
        res = res + (h / norm) * np.sinh(norm * eps) * SIGZ + (g / norm) * np.sinh(norm * eps) * SIGX
    return res


def _ising_u2(eps: complex, pos: int, L: int) -> np.ndarray:
    """isingU2MPO (IsingHamiltonian.cpp:169-201): exp(eps sz sz) split on a bond-2 MPO."""
    Z = np.zeros((3, 2, 2), dtype=np.complex128)
    Z[0], Z[1], Z[2] = SIG0, SIGZ, SIGX
    eps = complex(eps)
    if eps == 0:
        return SIG0.reshape(2, 1, 2, 1)
    D = 2
    if pos != 0 and pos != L - 1:
        C = np.zeros((D, D, 3), dtype=np.complex128)
        C[0, 0, 0] = np.cosh(eps)
        C[1, 1, 0] = np.sinh(eps)
        C[0, 1, 1] = np.sqrt(np.cosh(eps) * np.sinh(eps))
        C[1, 0, 1] = np.sqrt(np.cosh(eps) * np.sinh(eps))
        Dl, Dr = D, D
    else:
        C = np.zeros((1, D, 3), dtype=np.complex128)
        C[0, 0, 0] = np.sqrt(np.cosh(eps))
        C[0, 1, 1] = np.sqrt(np.sinh(eps))
        Dl, Dr = (1, D) if pos == 0 else (D, 1)
        C = C.reshape(Dl, Dr, 3, order="F")
    return _w_from_coeffs(C, Z)


def ising_umpo(L: int, J: float, g: float, h: float, delta: float, imag: bool) -> list:
    """IsingHamiltonian::getUMPO + constructU2T (IsingHamiltonian.cpp:131-148,
    220-244): 2nd-order Trotter U = e^{eps/2 H1} e^{eps H2} e^{eps/2 H1},
    eps = -delta (imaginary time) or -i delta (real time)."""
    eps = complex(-delta) if imag else -1j * delta
    ops = []
    for k in range(L):
        if 1 < k < L - 1:
            ops.append(ops[k - 1])
            continue
        U1 = _ising_u1(0.5 * eps, g, h)
        U2 = _ising_u2(J * eps, k, L)
        d, Dl, _, Dr = U2.shape
        res = U1 @ U2.reshape(d, Dl * d * Dr, order="F")
        res = res.reshape(d * Dl, d, Dr, order="F").transpose(0, 2, 1).reshape(d * Dl * Dr, d, order="F")
        res = res @ U1
        res = res.reshape(d * Dl, Dr, d, order="F").transpose(0, 2, 1).reshape(d, Dl, d, Dr, order="F")
        ops.append(np.ascontiguousarray(res))
    return ops


def schwinger_hmpo(N: int, mu: float, x: float, l0: float = 0.0, alpha: float = 0.0,
                   offset: float = 0.0, nu: float = 0.0, y: float = 1.0) -> list:
    """SchwingerHamiltonian::initHMPO (SchwingerHamiltonian.cpp:43-121): spin
    formulation, staggered fermions, gauge field integrated out, MPO bond 5."""
    Z = np.zeros((4, 2, 2), dtype=np.complex128)
    Z[0], Z[1], Z[2], Z[3] = SIG0, SIGX, SIGY_SCHW, SIGZ
    D = 5
    alpha_ = alpha + l0
    alphas = np.zeros(N)
    for k in range(N):
        signo = 1.0 if (k + 1) % 2 == 0 else -1.0
        alphas[k] = alpha_ - 0.25 * (1.0 - signo)
    sumA = np.zeros(N)
    tot = 0.0
    for k in range(N - 2, -1, -1):
        tot = tot + alphas[k]
        sumA[k] = tot
    gw = y
    ops = []
    for k in range(N):
        Dl = 1 if k == 0 else D
        Dr = 1 if k == N - 1 else D
        C = np.zeros((Dl, Dr, 4), dtype=np.complex128)
        if k != N - 1:
            C[0, 0, 0] = 1.0
        if k != 0:
            C[D - 1, Dr - 1, 0] = 1.0
        if 0 < k < N - 2:
            C[3, 3, 0] = 1.0
        ak = alphas[k]
        signok = 1.0 if (k + 1) % 2 == 0 else -1.0
        if k != N - 1:
            C[0, Dr - 1, 0] = gw * ak * ak + (gw * (k + 1) / 4.0 + mu / 2.0 + nu / 2.0 + offset / N)
            C[0, Dr - 1, 3] = (signok * mu / 2.0 + nu / 2.0) + gw * sumA[k]
        else:
            C[0, Dr - 1, 0] = mu / 2.0 + nu / 2.0 + offset / N
            C[0, Dr - 1, 3] = signok * mu / 2.0 + nu / 2.0
        if k != N - 1:
            C[0, 1, 1] = math.sqrt(x / 2)
            C[0, 2, 2] = math.sqrt(x / 2)
            if k < N - 2:
                C[0, 3, 3] = gw
            if k != 0:
                C[1, 4, 1] = math.sqrt(x / 2)
                C[2, 4, 2] = math.sqrt(x / 2)
                C[3, 4, 3] = (N - k - 1) / 2.0
        else:
            C[1, 0, 1] = math.sqrt(x / 2)
            C[2, 0, 2] = math.sqrt(x / 2)
        ops.append(_w_from_coeffs(C, Z))
    return ops


def identity_mpo(L: int, d: int = 2) -> list:
    return [SIG0.reshape(d, 1, d, 1).astype(np.complex128) for _ in range(L)]


# ---------------------------------------------------------------------------
# Contractions (wrapper/multipliers/TensorMultiplier.cpp, core/cpp/Operator.cpp)
# ---------------------------------------------------------------------------


def heff_apply(L: np.ndarray, W: np.ndarray, R: np.ndarray, A: np.ndarray) -> np.ndarray:
    """TensorMultiplier::product (TensorMultiplier.cpp:61-93) on a site-shaped
    tensor: y[s',a',r'] = sum L[a',b,a] W[s',b,s,c] R[r',c,r] A[s,a,r]."""
    t1 = np.tensordot(L, A, axes=([2], [1]))           # a' b s r
    t2 = np.tensordot(t1, W, axes=([1, 2], [1, 2]))    # a' r s' c
    y = np.tensordot(t2, R, axes=([1, 3], [2, 1]))     # a' s' r'
    return np.ascontiguousarray(y.transpose(1, 0, 2))


def heff_matvec(L, W, R, x: np.ndarray, offset: float = 0.0) -> np.ndarray:
    """TensorMultiplierOffset::product (TensorMultiplierOffset.cpp:14-17) on
    the column-major vector x; returns a vector of the same layout."""
    du, dd = W.shape[0], W.shape[2]
    A = x.reshape(dd, L.shape[2], R.shape[2], order="F")
    y = heff_apply(L, W, R, A).ravel(order="F")
    if offset:
        y = y + offset * x
    return y


def dagger_env(E: np.ndarray) -> np.ndarray:
    """permute(3,2,1) + conjugate (TensorMultiplierHermitian.cpp:21,25)."""
    return np.conj(E.transpose(2, 1, 0))


def dagger_op(W: np.ndarray) -> np.ndarray:
    """permute(3,2,1,4) + conjugate (TensorMultiplierHermitian.cpp:23)."""
    return np.conj(W.transpose(2, 1, 0, 3))


def heff_matvec_hermitian(L, W, R, x, offset: float = 0.0) -> np.ndarray:
    """TensorMultiplierHermitian(Offset)::product: 0.5 (H x + H^dagger x)
    (TensorMultiplierHermitian.cpp:37-70)."""
    y = 0.5 * (heff_matvec(L, W, R, x) + heff_matvec(dagger_env(L), dagger_op(W), dagger_env(R), x))
    if offset:
        y = y + offset * x
    return y


def heff_dense(L, W, R) -> np.ndarray:
    """TensorMultiplier::getFullTensor (TensorMultiplier.cpp:102-117):
    M[(s',a',r'),(s,a,r)] column-major on both sides."""
    M = np.einsum("pba,tbsc,qcr->tpqsar", L, W, R)
    n = M.shape[0] * M.shape[1] * M.shape[2]
    return M.reshape(n, n, order="F")


def env_left(Lold, ket, W, bra) -> np.ndarray:
    """Operator::contractleftop (Operator.cpp:273-322):
    Lnew[r, c, r'] = sum conj(bra[t,a',r]) Lold[a',b,a] W[t,b,s,c] ket[s,a,r']."""
    t1 = np.tensordot(Lold, ket, axes=([2], [1]))          # a' b s r'
    t2 = np.tensordot(t1, W, axes=([1, 2], [1, 2]))        # a' r' t c
    out = np.tensordot(np.conj(bra), t2, axes=([0, 1], [2, 0]))  # r r' c
    return np.ascontiguousarray(out.transpose(0, 2, 1))


def env_right(Rold, ket, W, bra) -> np.ndarray:
    """Operator::contractrightop (Operator.cpp:336-387):
    Rnew[l, b, l'] = sum conj(bra[t,l,r]) Rold[r,c,q] W[t,b,s,c] ket[s,l',q]."""
    t1 = np.tensordot(ket, Rold, axes=([2], [2]))          # s l' r c
    t2 = np.tensordot(t1, W, axes=([0, 3], [2, 3]))        # l' r t b
    out = np.tensordot(np.conj(bra), t2, axes=([0, 2], [2, 1]))  # l l' b
    return np.ascontiguousarray(out.transpose(0, 2, 1))


def norm_left(Lold, ket, bra) -> np.ndarray:
    """Contractor::contractL (Contractor.cpp:808-828): (Dr_bra, Dr_ket)."""
    return np.einsum("sar,ab,sbq->rq", np.conj(bra), Lold, ket)


def norm_right(Rold, ket, bra) -> np.ndarray:
    """Contractor::contractR (Contractor.cpp:830-848): (Dl_bra, Dl_ket)."""
    return np.einsum("slr,rq,smq->lm", np.conj(bra), Rold, ket)


def mbra_id(Lnorm, bra, Rnorm) -> np.ndarray:
    """Contractor::contractMbraId (Contractor.cpp:880-903): row vector
    v[s,l',r'] = sum conj(bra[s,l,r]) Lnorm[l,l'] Rnorm[r,r'] (ket layout)."""
    v = np.einsum("slr,lm,rq->smq", np.conj(bra), Lnorm, Rnorm)
    return v.ravel(order="F")


# ---------------------------------------------------------------------------
# Full-chain contractions (Contractor.cpp:467-556)
# ---------------------------------------------------------------------------


def contract_op(ket: MPS, ops: list, bra: MPS) -> complex:
    """Contractor::contract(ket, ops, bra) = <bra|ops|ket> incl. norm factors."""
    E = np.ones((1, 1, 1), dtype=np.complex128)
    for k in range(ket.L):
        E = env_left(E, ket.sites[k], ops[k], bra.sites[k])
    return complex(ket.normfact * bra.normfact * E.reshape(-1)[0])


def contract_overlap(ket: MPS, bra: MPS) -> complex:
    """Contractor::contract(ket, bra) = <bra|ket> incl. norm factors."""
    E = np.ones((1, 1), dtype=np.complex128)
    for k in range(ket.L):
        E = norm_left(E, ket.sites[k], bra.sites[k])
    return complex(ket.normfact * bra.normfact * E.reshape(-1)[0])


def doubled_mpo(ops: list) -> list:
    """The operator O^dag O as an MPO: (O^dag O)(s', b1 b2, s, c1 c2) =
    sum_t conj(O(t, b1, s', c1)) O(t, b2, s, c2), bond index b1 + wl b2."""
    out = []
    for W in ops:
        du, wl, dd, wr = W.shape
        X = np.einsum("tbpc,tqse->pbqsce", W.conj(), W)           # (s', b1, b2, s, c1, c2)
        out.append(X.reshape(dd, wl * wl, dd, wr * wr, order="F"))
    return out


def contract2(ops: list, ket: MPS, bra: MPS = None) -> complex:
    """Contractor::contract2(bra, ops, ket) = <bra|ops^dag ops|ket>
    (Contractor.cpp:634-718; contract2(ops, ket) when bra is ket)."""
    return contract_op(ket, doubled_mpo(ops), bra if bra is not None else ket)


def optimize_error(ops: list, orig: MPS, init: MPS):
    """errN and errT of Contractor::optimize (Contractor.cpp:263-276)."""
    norm0 = contract2(ops, orig).real
    norm1 = contract_overlap(init, init).real
    cross = contract_op(orig, ops, init)
    return norm0 + norm1 - 2 * cross.real, norm0


# ---------------------------------------------------------------------------
# QR / LQ gauge moves (core/cpp/Site.cpp:179-283, core/cpp/MPS.cpp:306-419)
# ---------------------------------------------------------------------------


def qr_reduced(M: np.ndarray):
    """wrapper::qr (wrapper/qr.cpp:33-110): Q (m x K), R (K x n), K=min(m,n)."""
    return np.linalg.qr(M, mode="reduced")


def lq_reduced(M: np.ndarray):
    """wrapper::lq (wrapper/qr.cpp:112-188): L (m x K), Q (K x n)."""
    q, r = np.linalg.qr(M.conj().T, mode="reduced")
    return r.conj().T, q.conj().T


def site_gauge_r(A: np.ndarray, left=None):
    """Site::gaugeR with cutD=0 (Site.cpp:179-208); ``left`` is absorbed
    first (reduceDimR, Site.cpp:240-261).  Returns (newA, rightterm)."""
    if left is not None:
        A = site_reduce_r(A, left)
    d, Dl, Dr = A.shape
    Q, R = qr_reduced(A.reshape(d * Dl, Dr, order="F"))
    K = Q.shape[1]
    A = Q.reshape(d, Dl, K, order="F")
    if K == 1 and R.shape[1] == 1:
        aux = R[0, 0]
        phase = aux / abs(aux) if abs(aux) != 0 else 1.0
        A = A * phase
        R = np.array([[abs(aux)]], dtype=np.complex128)
    return A, R


def site_gauge_l(A: np.ndarray, right=None):
    """Site::gaugeL with cutD=0 (Site.cpp:210-238). Returns (newA, leftterm)."""
    if right is not None:
        A = site_reduce_l(A, right)
    d, Dl, Dr = A.shape
    M = A.transpose(1, 0, 2).reshape(Dl, d * Dr, order="F")
    Lm, Q = lq_reduced(M)
    K = Q.shape[0]
    A = Q.reshape(K, d, Dr, order="F").transpose(1, 0, 2)
    if K == 1 and Lm.shape[0] == 1:
        aux = Lm[0, 0]
        phase = aux / abs(aux) if abs(aux) != 0 else 1.0
        A = A * phase
        Lm = np.array([[abs(aux)]], dtype=np.complex128)
    return np.ascontiguousarray(A), Lm


def site_reduce_r(A: np.ndarray, left: np.ndarray) -> np.ndarray:
    """Site::reduceDimR (Site.cpp:240-261): A <- left * A on the Dl leg."""
    if left.size == 1:
        return left.reshape(-1)[0] * A
    return np.ascontiguousarray(np.einsum("ka,sar->skr", left, A))


def site_reduce_l(A: np.ndarray, right: np.ndarray) -> np.ndarray:
    """Site::reduceDimL (Site.cpp:263-283): A <- A * right on the Dr leg."""
    if right.size == 1:
        return right.reshape(-1)[0] * A
    return np.ascontiguousarray(np.einsum("sar,rk->sak", A, right))


def gauge_cond_all(mps: MPS, direction: str, normal: bool = True) -> None:
    """MPS::gaugeCond(dir, normal, cutD=0) (MPS.cpp:306-364)."""
    tmp = np.ones((1, 1), dtype=np.complex128)
    if direction == "L":
        for pos in range(mps.L - 1, -1, -1):
            mps.sites[pos], tmp = site_gauge_l(mps.sites[pos], tmp)
        mps.gauge = 1
    else:
        for pos in range(mps.L):
            mps.sites[pos], tmp = site_gauge_r(mps.sites[pos], tmp)
        mps.gauge = 2
    mps.bond = min(mps.bond or 10 ** 9, mps.max_bond())
    if normal:
        mps.normfact = 1.0
    else:
        mps.normfact = mps.normfact * abs(tmp.reshape(-1)[0])


def gauge_cond_site(mps: MPS, pos: int, direction: str, nxt: bool = False) -> None:
    """MPS::gaugeCond(pos, dir, next) (MPS.cpp:366-419)."""
    old = mps.sites[pos].shape
    if direction == "L":
        mps.sites[pos], tmp = site_gauge_l(mps.sites[pos])
        if (mps.sites[pos].shape[1] != old[1] or nxt) and pos > 0:
            mps.sites[pos - 1] = site_reduce_l(mps.sites[pos - 1], tmp)
        if pos == 0 and nxt:
            mps.normfact *= abs(tmp.reshape(-1)[0])
    else:
        mps.sites[pos], tmp = site_gauge_r(mps.sites[pos])
        if pos < mps.L - 1 and (mps.sites[pos].shape[2] != old[2] or nxt):
            mps.sites[pos + 1] = site_reduce_r(mps.sites[pos + 1], tmp)
        if nxt and pos == mps.L - 1:
            mps.normfact *= abs(tmp.reshape(-1)[0])
    mps.gauge = 0


def increase_bond_dimension(mps: MPS, D: int) -> None:
    """MPS::increaseBondDimensionWithNoise(D, 0) (MPS.cpp:654-719): integer
    bond schedule and zero padding (Site::changeDimensions, mwArray::resize)."""
    if D <= mps.bond:
        return
    L = mps.L
    cumd = 1
    cumdr_last = 1
    boundR = L - 1
    done = False
    while not done and boundR > 0:
        dim = mps.sites[boundR].shape[0]
        if cumdr_last * dim < D:
            boundR -= 1
            cumdr_last *= dim
        else:
            done = True
    cumdr = D if boundR > 0 else cumdr_last * mps.sites[0].shape[0]
    maxbond = 1
    for k in range(L):
        old = mps.sites[k].shape
        if k == 0:
            newDl = old[1]
        else:
            newDl = min(cumd, cumdr) if (cumd < D or cumdr < D) else D
        posd = mps.sites[k].shape[0]
        if cumd < D:
            cumd *= posd
        if k == boundR:
            cumdr = cumdr_last
        elif k > boundR:
            cumdr = cumdr // posd
        if k == L - 1:
            newDr = old[2]
        else:
            newDr = min(cumd, cumdr) if (cumd < D or cumdr < D) else D
        a = np.zeros((old[0], newDl, newDr), dtype=np.complex128)
        m1, m2 = min(old[1], newDl), min(old[2], newDr)
        a[:, :m1, :m2] = mps.sites[k][:, :m1, :m2]
        mps.sites[k] = a
        maxbond = max(maxbond, newDl, newDr)
    mps.bond = maxbond
    mps.gauge = 0


# ---------------------------------------------------------------------------
# Local eigensolver
# ---------------------------------------------------------------------------

LOWEST_PRIMME = 801  # Contractor.cpp:29


def lowest_eigpair(matvec, n: int, x0: np.ndarray, dense=None, tol: float = 1e-12,
                   max_krylov: int = 64, max_restarts: int = 60):
    """Contractor::solveEigs (Contractor.cpp:3067-3138): below LOWEST_PRIMME the
    reference diagonalises the dense, hermitised matrix (wrapper::eig); above
    it calls PRIMME, here restated as restarted Lanczos with full
    reorthogonalisation and ||r|| <= tol * max|Ritz| convergence."""
    if dense is not None and n < LOWEST_PRIMME:
        M = dense()
        M = 0.5 * (M + M.conj().T)
        w, v = np.linalg.eigh(M)
        return float(w[0]), v[:, 0].copy()
    x = x0.astype(np.complex128).copy()
    nx = np.linalg.norm(x)
    x = x / nx if nx > 0 else np.full(n, 1 / math.sqrt(n), dtype=np.complex128)
    m = min(n, max_krylov)
    theta = 0.0
    V = np.empty((m, n), dtype=np.complex128)  # basis rows, filled in place
    for _ in range(max_restarts):
        V[0] = x
        a, b = [], []
        conv = False
        for j in range(m):
            w = matvec(V[j])
            a.append(float(np.vdot(V[j], w).real))
            w = w - a[j] * V[j]
            if j > 0:
                w = w - b[j - 1] * V[j - 1]
            Vm = V[: j + 1]
            for _p in range(2):
                w = w - Vm.T @ (Vm.conj() @ w)
            beta = float(np.linalg.norm(w))
            b.append(beta)
            T = np.diag(a) + np.diag(b[:-1], 1) + np.diag(b[:-1], -1)
            ev, es = np.linalg.eigh(T)
            theta, s = float(ev[0]), es[:, 0]
            scale = max(abs(ev[0]), abs(ev[-1]))
            if beta * abs(s[-1]) <= tol * scale or beta <= 1e-14 * scale or j + 1 == n:
                conv = True
                break
            if j + 1 < m:
                V[j + 1] = w / beta
        y = V[: len(a)].T @ s
        x = y / np.linalg.norm(y)
        if conv:
            break
    return theta, x


# ---------------------------------------------------------------------------
# Environment cache (core/cpp/TmpManager.cpp) and the sweeps
# ---------------------------------------------------------------------------


class EnvCache:
    """TmpManager (TmpManager.cpp:22-160): operL[0] = operR[L-1] = 1 and
    validity flags; entries are filled recursively (Contractor.cpp:723-764)."""

    def __init__(self, L: int):
        self.L = L
        self.opL = [None] * L
        self.opR = [None] * L
        self.opL[0] = np.ones((1, 1, 1), dtype=np.complex128)
        self.opR[L - 1] = np.ones((1, 1, 1), dtype=np.complex128)
        self.okL = [False] * L
        self.okR = [False] * L
        self.okL[0] = True
        self.okR[L - 1] = True
        self.norms = []  # per level: [normL list, normR list, okL, okR]

    def outofdate_l(self, l):
        if l > 0:
            self.okL[l] = False

    def outofdate_r(self, l):
        if l < self.L - 1:
            self.okR[l] = False

    def left(self, pos, ops, ket, bra):
        if not self.okL[pos]:
            self.left(pos - 1, ops, ket, bra)
            self.opL[pos] = env_left(self.opL[pos - 1], ket.sites[pos - 1], ops[pos - 1], bra.sites[pos - 1])
            self.okL[pos] = True
        return self.opL[pos]

    def right(self, pos, ops, ket, bra):
        if not self.okR[pos]:
            self.right(pos + 1, ops, ket, bra)
            self.opR[pos] = env_right(self.opR[pos + 1], ket.sites[pos + 1], ops[pos + 1], bra.sites[pos + 1])
            self.okR[pos] = True
        return self.opR[pos]


@dataclass
class SweepStats:
    rounds: int = 0
    site_solves: int = 0
    matvecs: int = 0
    energies: list = field(default_factory=list)


def _prepare_init(mps: MPS, D: int) -> None:
    """Common prologue of findGroundState / optimize (Contractor.cpp:1359-1373)."""
    if D > 0:
        if D > mps.bond:
            increase_bond_dimension(mps, D)
        elif D < mps.bond:
            truncated = truncate_mps(mps, D)
            mps.sites, mps.normfact, mps.bond, mps.gauge = (
                truncated.sites, truncated.normfact, truncated.bond, truncated.gauge)
    gauge_cond_all(mps, "R", True)
    gauge_cond_all(mps, "L", True)


def find_ground_state(ops: list, D: int, mps: MPS, offset: float = 0.0,
                      convtol: float = 1e-5, eigtol: float = 0.0, stats: SweepStats = None):
    """Contractor::findGroundState (Contractor.cpp:1352-1533), single-site
    DMRG sweeping 0 -> L-1 -> 0 ...; returns the energy."""
    st = stats if stats is not None else SweepStats()
    L = mps.L
    _prepare_init(mps, D)
    cache = EnvCache(L)
    energy = contract_op(mps, ops, mps).real
    val = energy
    right, pos, rnd, done = True, 0, 0, False
    tol = eigtol if eigtol > 0 else 1e-12
    while not done:
        Lenv = cache.left(pos, ops, mps, mps)
        Renv = cache.right(pos, ops, mps, mps)
        W = ops[pos]
        A = mps.sites[pos]
        n = A.size
        count = [0]

        def mv(v, L_=Lenv, W_=W, R_=Renv):
            count[0] += 1
            return heff_matvec(L_, W_, R_, v, offset)

        theta, U = lowest_eigpair(
            mv, n, A.ravel(order="F"),
            dense=lambda: heff_dense(Lenv, W, Renv) + offset * np.eye(n), tol=tol)
        st.matvecs += count[0]
        st.site_solves += 1
        val = theta - offset
        mps.sites[pos] = U.reshape(A.shape, order="F")
        if (val - energy > 1e-8) and (val - energy > abs(energy + offset) * 1e-10):
            if val - energy > abs(energy + offset) * convtol:
                raise RuntimeError("energy increasing (Contractor.cpp:1418-1427 exit 212)")
        gauge_cond_site(mps, pos, "R" if right else "L", True)
        for l in range(pos + 1, L):
            cache.outofdate_l(l)
        for l in range(pos - 1, -1, -1):
            cache.outofdate_r(l)
        if right:
            if pos == L - 1:
                right = False
                done = abs(energy - val) < convtol * abs(energy + offset)
                if not done and abs(val) < 1e-13:
                    done = True
                energy = val
                st.energies.append(val)
                if not done:
                    gauge_cond_site(mps, pos, "L", True)
                    pos -= 1
                rnd += 1
            else:
                pos += 1
        else:
            if pos == 0:
                right = True
                done = abs(energy - val) < convtol * abs(energy + offset)
                if not done and abs(val) < 1e-13:
                    done = True
                energy = val
                st.energies.append(val)
                if not done:
                    gauge_cond_site(mps, pos, "R", True)
                    pos += 1
                rnd += 1
            else:
                pos -= 1
    st.rounds = rnd
    return energy


def heff2_apply(L: np.ndarray, W1: np.ndarray, W2: np.ndarray, R: np.ndarray, T: np.ndarray) -> np.ndarray:
    """Two-site effective Hamiltonian on Theta[s1, s2, a, r]:
    y[s1',s2',a',r'] = sum L[a',b,a] W1[s1',b,s1,c] W2[s2',c,s2,e] R[r',e,r] T[s1,s2,a,r]."""
    return np.einsum("pba,ubsc,vcte,qer,star->uvpq", L, W1, W2, R, T, optimize=True)


def find_ground_state_two_site(ops: list, D: int, mps: MPS, offset: float = 0.0, convtol: float = 1e-5,
                               eigtol: float = 0.0, stats: SweepStats = None):
    """Two-site DMRG as the library runs it (no counterpart in the reference,
    whose sweeps are single site): start from gaugeCond('R',1) then
    gaugeCond('L',1) (after a cut to D if the state is larger), optimise the
    bond (pos, pos+1) with the lowest eigenpair of the two-site H_eff, split
    by svd_cut(Theta, D) with the singular values moved in the sweep
    direction, and at a chain end solve the same bond again in the other
    direction.  Convergence |E_old - E_new| < convtol |E + offset| at the
    ends.  Returns (energy, max relative discarded weight)."""
    st = stats if stats is not None else SweepStats()
    L = mps.L
    if D < mps.bond:
        t = truncate_mps(mps, D)
        mps.sites, mps.normfact = t.sites, t.normfact
        mps.bond = t.max_bond()
    gauge_cond_all(mps, "R", True)
    gauge_cond_all(mps, "L", True)
    cache = EnvCache(L)
    energy = contract_op(mps, ops, mps).real
    val, dmax = energy, 0.0
    right, pos, rnd, done = True, 0, 0, False
    tol = eigtol if eigtol > 0 else 1e-12
    while not done:
        Lenv = cache.left(pos, ops, mps, mps)
        Renv = cache.right(pos + 1, ops, mps, mps)
        A1, A2 = mps.sites[pos], mps.sites[pos + 1]
        d1, Dl, _ = A1.shape
        d2, _, Dr = A2.shape
        T = np.einsum("sam,tmr->star", A1, A2)
        shape = T.shape
        n = T.size

        def mv(v, L_=Lenv, R_=Renv, W1=ops[pos], W2=ops[pos + 1]):
            st.matvecs += 1
            return (heff2_apply(L_, W1, W2, R_, v.reshape(shape, order="F")).ravel(order="F")
                    + offset * v)

        def dense():
            return np.array([mv(e) for e in np.eye(n, dtype=np.complex128)]).T

        theta, x = lowest_eigpair(mv, n, T.ravel(order="F"), dense=dense if n <= 128 else None, tol=tol)
        st.site_solves += 1
        val = theta - offset
        T = x.reshape(shape, order="F")
        M = T.transpose(0, 2, 1, 3).reshape(d1 * Dl, d2 * Dr, order="F")      # rows (s1, a), cols (s2, r)
        U, s, Vh, w = svd_cut(M, D)
        tot = float(np.sum(np.linalg.svd(M, compute_uv=False) ** 2))
        dmax = max(dmax, w / tot if tot > 0 else 0.0)
        K = s.size
        if right:
            left, rightf = U, s[:, None] * Vh
        else:
            left, rightf = U * s[None, :], Vh
        mps.sites[pos] = np.ascontiguousarray(left.reshape(d1, Dl, K, order="F"))
        mps.sites[pos + 1] = np.ascontiguousarray(
            rightf.reshape(K, d2, Dr, order="F").transpose(1, 0, 2))
        for l in range(pos + 1, L):
            cache.outofdate_l(l)
        for l in range(pos, -1, -1):
            cache.outofdate_r(l)
        if (right and pos == L - 2) or (not right and pos == 0):
            done = abs(energy - val) < convtol * abs(energy + offset)
            if not done and abs(val) < 1e-13:
                done = True
            energy = val
            right = not right
            rnd += 1
        else:
            pos += 1 if right else -1
    st.rounds += rnd
    mps.normfact = 1.0
    mps.bond = mps.max_bond()
    return energy, dmax


def find_next_excited_state(ops: list, D: int, levels: list, mps: MPS, offset: float = 0.0,
                            convtol: float = 1e-5, eigtol: float = 0.0, excorthtol: float = 0.0,
                            stats: SweepStats = None):
    """Contractor::findNextExcitedState (Contractor.cpp:2676-2727): penalty
    max(20 (maxE - minE), |offset|), or L/2 for a single level, then
    findGroundStateWithProjectorPenalty."""
    nextK = len(levels)
    energies = [contract_op(lv, ops, lv).real + offset for lv in levels]
    minE, maxE = min(energies), max(energies)
    newOffset = max(20 * (maxE - minE), abs(offset))
    if nextK == 1 or newOffset < 1e-6:
        newOffset = levels[0].L * 0.5
    pens = [newOffset] * nextK
    while True:
        e = find_gs_with_projector_penalty(ops, D, pens, levels, mps, offset, convtol, eigtol, stats)
        if excorthtol <= 0:
            return e
        again = False
        for k, lv in enumerate(levels):
            if abs(contract_overlap(mps, lv)) > excorthtol:
                pens[k] *= 2
                again = True
        if not again:
            return e


MAX_ROUND_EXCTD = 1000  # Contractor.cpp:26


def find_gs_with_projector_penalty(ops, D, pens, levels, mps: MPS, offset=0.0, convtol=1e-5,
                                   eigtol=0.0, stats: SweepStats = None):
    """Contractor::findGroundStateWithProjectorPenalty (Contractor.cpp:2739-2956)
    with TensorMultiplierProjMulti(hermitian=true) (TensorMultiplierProjMulti.cpp:81-90)."""
    st = stats if stats is not None else SweepStats()
    L = mps.L
    _prepare_init(mps, D)
    nextK = len(levels)
    energy = contract_op(mps, ops, mps).real + offset
    for k in range(nextK):
        ov = contract_overlap(mps, levels[k])
        energy += pens[k] * abs(ov) ** 2
    energy -= offset
    cache = EnvCache(L)
    # normL[k][pos] (D_level x D_init), normR[k][pos]
    nL = [[None] * L for _ in range(nextK)]
    nR = [[None] * L for _ in range(nextK)]
    for k in range(nextK):
        nL[k][0] = np.ones((1, 1), dtype=np.complex128)
        nR[k][L - 1] = np.ones((1, 1), dtype=np.complex128)

    def calc_l(pos):
        if not cache.okL[pos]:
            calc_l(pos - 1)
            cache.opL[pos] = env_left(cache.opL[pos - 1], mps.sites[pos - 1], ops[pos - 1], mps.sites[pos - 1])
            for k in range(nextK):
                nL[k][pos] = norm_left(nL[k][pos - 1], mps.sites[pos - 1], levels[k].sites[pos - 1])
            cache.okL[pos] = True

    def calc_r(pos):
        if not cache.okR[pos]:
            calc_r(pos + 1)
            cache.opR[pos] = env_right(cache.opR[pos + 1], mps.sites[pos + 1], ops[pos + 1], mps.sites[pos + 1])
            for k in range(nextK):
                nR[k][pos] = norm_right(nR[k][pos + 1], mps.sites[pos + 1], levels[k].sites[pos + 1])
            cache.okR[pos] = True

    val = energy
    right, pos, rnd, done = True, 0, 0, False
    tol = eigtol if eigtol > 0 else 1e-12
    while not done:
        calc_l(pos)
        calc_r(pos)
        Lenv, Renv, W = cache.opL[pos], cache.opR[pos], ops[pos]
        A = mps.sites[pos]
        n = A.size
        vecs = [mbra_id(nL[k][pos], levels[k].sites[pos], nR[k][pos]) for k in range(nextK)]
        count = [0]

        def mv(v):
            count[0] += 1
            y = heff_matvec_hermitian(Lenv, W, Renv, v)
            for k in range(nextK):
                y = y + pens[k] * (vecs[k] @ v) * vecs[k].conj()
            return y + offset * v

        def dense():
            M = heff_dense(Lenv, W, Renv)
            for k in range(nextK):
                M = M + pens[k] * np.outer(vecs[k].conj(), vecs[k])
            return M + offset * np.eye(n)

        theta, U = lowest_eigpair(mv, n, A.ravel(order="F"), dense=dense, tol=tol)
        st.matvecs += count[0]
        st.site_solves += 1
        val = theta - offset
        mps.sites[pos] = U.reshape(A.shape, order="F")
        if (val - energy > 1e-8) and (val - energy > abs(energy + offset) * 1e-10):
            if val - energy > abs(energy + offset) * 1e-6:
                raise RuntimeError("energy increasing (Contractor.cpp:2842-2853 exit 212)")
        gauge_cond_site(mps, pos, "R" if right else "L", True)
        for l in range(pos + 1, L):
            cache.outofdate_l(l)
        for l in range(pos - 1, -1, -1):
            cache.outofdate_r(l)
        at_end = (right and pos == L - 1) or ((not right) and pos == 0)
        if at_end:
            done = abs(energy - val) < convtol * abs(energy + offset)
            if not done and (abs(energy - val) < 1e-12 or rnd > MAX_ROUND_EXCTD):
                done = True
            energy = val
            st.energies.append(val)
            if not done:
                if right:
                    gauge_cond_site(mps, pos, "L", True)
                    pos -= 1
                else:
                    gauge_cond_site(mps, pos, "R", True)
                    pos += 1
            right = not right
            rnd += 1
        else:
            pos += 1 if right else -1
    st.rounds = rnd
    return energy


def check_distance_convergence(distance: float, c1: complex, c2: complex, normA: float,
                               normB: float, convtol: float):
    """Contractor::checkDistanceConvergence (Contractor.cpp:940-999)."""
    newd = normA * (normA * c1.real - 2 * c2.real) + normB * normB
    if math.isnan(newd):
        raise RuntimeError("NaN distance (Contractor.cpp:954-960 exit 1)")
    if (newd - distance) > convtol * abs(distance):
        if abs(newd) > convtol and abs(newd - distance) > 1e-12:
            raise RuntimeError("distance increasing (Contractor.cpp:963-975 exit 212)")
        done = True
    if abs((distance - newd) / distance) < convtol:
        done = True
    else:
        done = False
    if (abs(distance) + abs(newd)) * convtol < 1e-14:
        if abs(distance - newd) < convtol:
            done = True
    return done, newd


def optimize(ops: list, orig: MPS, init: MPS, D: int = 0, convtol: float = 1e-5,
             stats: SweepStats = None) -> None:
    """Contractor::optimize (Contractor.cpp:77-278): variational |init> ~ ops|orig>
    at fixed bond dimension; init is normalised, its normfact carries the norm."""
    st = stats if stats is not None else SweepStats()
    _prepare_init(init, D)
    L = orig.L
    cache = EnvCache(L)
    distance = abs(contract_overlap(orig, orig)) + abs(contract_overlap(init, init))
    right, pos, rnd, done = True, 0, 1, False
    c1 = c2 = 0
    while not done:
        Lenv = cache.left(pos, ops, orig, init)
        Renv = cache.right(pos, ops, orig, init)
        M = heff_apply(Lenv, ops[pos], Renv, orig.sites[pos])
        st.matvecs += 1
        nM = float(np.linalg.norm(M))
        init.sites[pos] = M / nM
        gauge_cond_site(init, pos, "R" if right else "L")
        A = init.sites[pos].ravel(order="F")
        c1 = complex(np.vdot(A, A))
        c2 = complex(np.vdot(A, M.ravel(order="F")))
        for l in range(pos + 1, L):
            cache.outofdate_l(l)
        for l in range(pos - 1, -1, -1):
            cache.outofdate_r(l)
        if right:
            if pos == L - 1:
                right = False
                done, distance = check_distance_convergence(distance, c1, c2, init.normfact,
                                                            orig.normfact, convtol)
                if not done:
                    gauge_cond_site(init, pos, "L")
                    if pos > 0:
                        pos -= 1
                rnd += 1
            else:
                pos += 1
        else:
            if pos == 0:
                right = True
                done, distance = check_distance_convergence(distance, c1, c2, init.normfact,
                                                            orig.normfact, convtol)
                if not done:
                    gauge_cond_site(init, pos, "R")
                    if pos < L - 1:
                        pos += 1
                rnd += 1
            else:
                pos -= 1
    init.normfact = c2.real / c1.real
    init.normfact = init.normfact * orig.normfact
    st.rounds += rnd


# ---------------------------------------------------------------------------
# Truncation, observables
# ---------------------------------------------------------------------------


def svd_cut(M: np.ndarray, cutD: int):
    """wrapper::svd(A, tol=0, nr=cutD, U, S, Vdagger) (wrapper/svd.cpp:23-118):
    thin SVD keeping the min(cutD, rank-dims) largest values; also returns the
    discarded weight sum_{i>=cut} s_i^2 (not returned by the reference)."""
    U, s, Vh = np.linalg.svd(M, full_matrices=False)
    nr = min(cutD, s.size) if cutD > 0 else s.size
    # tol = 0: values that are not > 0 are cut as well (svd.cpp:95-101)
    nr = int(np.sum(s[:nr] > 0.0))
    if nr == 0:
        raise ValueError("svd: no singular value above 0")
    disc = float(np.sum(s[nr:] ** 2))
    return U[:, :nr], s[:nr], Vh[:nr, :], disc


def truncate_mps(mps: MPS, D: int):
    """MPS(const MPS&, int D) (MPS.cpp:761-772) = gaugeCond('L', 0, D): right
    to left SVD cuts keeping the norm in normfact. Returns the new MPS and the
    discarded weights per bond as attribute ``discarded``."""
    out = mps.copy()
    tmp = np.ones((1, 1), dtype=np.complex128)
    disc = []
    for pos in range(out.L - 1, -1, -1):
        A = site_reduce_l(out.sites[pos], tmp)
        d, Dl, Dr = A.shape
        M = A.transpose(1, 0, 2).reshape(Dl, d * Dr, order="F")
        U, s, Vh, w = svd_cut(M, D)
        disc.append(w)
        tmp = U * s[None, :]
        K = Vh.shape[0]
        A = Vh.reshape(K, d, Dr, order="F").transpose(1, 0, 2)
        if K == 1 and tmp.shape[0] == 1:
            aux = tmp[0, 0]
            phase = aux / abs(aux) if abs(aux) != 0 else 1.0
            A = A * phase
            tmp = np.array([[abs(aux)]], dtype=np.complex128)
        out.sites[pos] = np.ascontiguousarray(A)
    out.gauge = 1
    out.bond = out.max_bond()
    out.normfact = out.normfact * abs(tmp.reshape(-1)[0])
    out.discarded = disc[::-1]
    return out


def _gauge_l_cut(A: np.ndarray, cutD: int):
    """Site::gaugeL with cutD > 0 (Site.cpp:210-238) on an already reduced
    site: SVD of A as (Dl x d Dr); returns (new site, leftterm, discarded)."""
    d, Dl, Dr = A.shape
    M = A.transpose(1, 0, 2).reshape(Dl, d * Dr, order="F")
    U, sv, Vh, w = svd_cut(M, cutD)
    left = U * sv[None, :]
    K = Vh.shape[0]
    A = Vh.reshape(K, d, Dr, order="F").transpose(1, 0, 2)
    if K == 1 and left.shape[0] == 1:
        aux = left[0, 0]
        phase = aux / abs(aux) if abs(aux) != 0 else 1.0
        A = A * phase
        left = np.array([[abs(aux)]], dtype=np.complex128)
    return np.ascontiguousarray(A), left, w


def _gauge_r_cut(A: np.ndarray, cutD: int):
    """Site::gaugeR with cutD > 0 (Site.cpp:179-208): SVD of A as (d Dl x Dr);
    returns (new site, rightterm, discarded)."""
    d, Dl, Dr = A.shape
    U, sv, Vh, w = svd_cut(A.reshape(d * Dl, Dr, order="F"), cutD)
    right = sv[:, None] * Vh
    K = U.shape[1]
    A = U.reshape(d, Dl, K, order="F")
    if K == 1 and right.shape[1] == 1:
        aux = right[0, 0]
        phase = aux / abs(aux) if abs(aux) != 0 else 1.0
        A = A * phase
        right = np.array([[abs(aux)]], dtype=np.complex128)
    return np.ascontiguousarray(A), right, w


def apply_mpo(ops: list, mps: MPS, cutD: int = 0, dagger: bool = False, direction: str = "L") -> MPS:
    """MPS::applyExactly (cutD <= 0) and MPS::truncate(ops, mps, cutD, dagger,
    dir) (MPS.cpp:858-936): each site contracted with its operator and the
    carried factor (Site::reduceDimLOp / reduceDimROp, Site.cpp:303-402),
    then gauged by an SVD cut (applyExactly cuts at the full dimension,
    Dl*w or Dr*w, which only drops zero values).  Returns a new MPS with
    attribute ``discarded`` (sum of dropped squares)."""
    out = mps.copy()
    L = out.L
    tmp = np.ones((1, 1), dtype=np.complex128)
    disc = 0.0
    order = range(L - 1, -1, -1) if direction == "L" else range(L)
    for pos in order:
        W = ops[pos]
        if dagger:
            W = W.transpose(2, 1, 0, 3).conj()
        du, wl, dd, wr = W.shape
        A = out.sites[pos]
        d, Dl, Dr = A.shape
        if direction == "L":
            cut = cutD if cutD > 0 else Dl * wl
            t = tmp.reshape(wr, Dr, -1, order="F")                  # (c, r, beta)
            An = np.einsum("ubsc,sar,crq->ubaq", W, A, t)           # (u, b, a, beta)
            An = An.reshape(du, wl * Dl, t.shape[2], order="F")     # left index b + wl a
            out.sites[pos], tmp, w = _gauge_l_cut(An, cut)
        else:
            cut = cutD if cutD > 0 else Dr * wr
            t = tmp.reshape(-1, wl, Dl, order="F")                  # (beta, b, a)
            An = np.einsum("qba,ubsc,sar->uqcr", t, W, A)           # (u, beta, c, r)
            An = An.reshape(du, t.shape[0], wr * Dr, order="F")     # right index c + wr r
            out.sites[pos], tmp, w = _gauge_r_cut(An, cut)
        disc += w
    if tmp.size != 1:
        raise ValueError("apply_mpo: final factor is not a scalar")
    out.normfact = mps.normfact * abs(tmp.reshape(-1)[0])
    out.gauge = 1 if direction == "L" else 2
    # applyExactly leaves the bond field alone; truncate lowers it to the
    # largest bond present (MPS.cpp:919,934)
    if cutD > 0:
        out.bond = min(mps.bond or out.max_bond(), out.max_bond())
    out.discarded = disc
    return out


def mps_to_vector(mps: MPS) -> np.ndarray:
    """Dense state vector (normfact included), index s_0 + d s_1 + d^2 s_2 ...
    (small L only)."""
    v = mps.sites[0][:, 0, :]                                      # (s0, r)
    for A in mps.sites[1:]:
        v = np.einsum("xa,sar->xsr", v, A).reshape(-1, A.shape[2], order="F")
    return mps.normfact * v[:, 0]


def expectation_values(mps: MPS, op2: np.ndarray) -> np.ndarray:
    """<op_k>/<psi|psi> for every site (programs/banulsm/curved/flatIsing.cpp:258-282)."""
    L = mps.L
    ident = identity_mpo(L)
    nrm = contract_overlap(mps, mps).real
    out = []
    for pos in range(L):
        ops = list(ident)
        ops[pos] = op2.reshape(2, 1, 2, 1).astype(np.complex128)
        out.append(contract_op(mps, ops, mps).real / nrm)
    return np.array(out)


def schmidt_values(mps: MPS, pos: int) -> np.ndarray:
    """Contractor::getSchmidtValues (Contractor.cpp:2243-2270): eigenvalues of
    the right-contracted density matrix after gaugeCond('R',1)."""
    L = mps.L
    if pos == L:
        return np.array([1.0])
    aux = mps.copy()
    if aux.gauge not in (2, 3):
        gauge_cond_all(aux, "R", True)
    if pos == 0:
        pos = L // 2
    E = np.ones((1, 1), dtype=np.complex128)
    for k in range(L - 1, pos - 1, -1):
        E = norm_right(E, aux.sites[k], aux.sites[k])
    Dm = aux.sites[pos].shape[1]
    E = E.reshape(Dm, Dm)
    return np.linalg.eigvalsh(0.5 * (E + E.conj().T))


def entropy(mps: MPS, pos: int) -> float:
    """Contractor::getEntropy (Contractor.cpp:2045-2076): -sum lam log2 lam over
    |lam| > 1e-12."""
    if pos == mps.L:
        return 0.0
    lam = schmidt_values(mps, pos)
    return float(sum(-t * math.log2(t) for t in lam if abs(t) > 1e-12))


# ---------------------------------------------------------------------------
# Independent checks: exact diagonalisation, free-fermion closed form
# ---------------------------------------------------------------------------


def mpo_dense(ops: list) -> np.ndarray:
    """Dense operator of an MPO (small L only), basis index sum_k s_k d^k."""
    T = ops[0][:, 0, :, :]            # s' s c
    for W in ops[1:]:
        T = np.einsum("xyb,tbsc->xtysc", T, W)
        a, b_, c_, e, f = T.shape
        T = T.reshape(a * b_, c_ * e, f, order="F")
    return T[:, :, 0]


def tfim_open_energy(L: int, J: float, g: float) -> float:
    """Ground energy of H = J sum sz_i sz_{i+1} + g sum sx_i, open chain, from
    free fermions (Lieb, Schultz, Mattis 1961; Pfeuty 1970): E0 = -sum_k eps_k
    with eps_k the singular values of the L x L bidiagonal matrix with g on
    the diagonal and J on the first superdiagonal."""
    B = np.diag(np.full(L, float(g))) + np.diag(np.full(L - 1, float(J)), 1)
    return -float(np.sum(np.linalg.svd(B, compute_uv=False)))
