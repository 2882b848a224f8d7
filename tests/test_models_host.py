"""MPO builders beyond Ising and Schwinger, checked on the CPU: the oracle's
restatement and the library's own host builder (models.cpp, compiled here
with g++) against the tensors the reference itself built (tests/golden),
and the Bose-Hubbard MPO against the Hamiltonian written out term by term."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import mps_oracle as mo

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# (name, L, N, t, U, Ntarget, penN, V): bh6 has exactly representable
# coefficient products (bit-exact whatever the summation order), bh6x not
BH = [("bh6", 6, 2, 1.0, 2.0, 3, 0.25, 0.5), ("bh6x", 6, 3, 0.7, 1.3, 4, 0.3, 0.15)]


@pytest.fixture(scope="module")
def dump_bin(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("models") / "models_dump"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "mpsdyn_b200", "csrc"), "-o", str(out),
                    os.path.join(HERE, "native", "models_dump.cpp"),
                    os.path.join(ROOT, "mpsdyn_b200", "csrc", "models.cpp")], check=True)
    return str(out)


def library_bh(dump_bin, *args):
    lines = subprocess.run([dump_bin, *[str(a) for a in args]], capture_output=True, text=True,
                           check=True).stdout.strip().split("\n")
    ws = []
    for line in lines:
        v = line.split()
        dims = [int(x) for x in v[:4]]
        z = np.array([float(x) for x in v[4:]]).reshape(-1, 2)
        ws.append((z[:, 0] + 1j * z[:, 1]).reshape(dims, order="F"))
    return ws


@pytest.mark.parametrize("name,L,N,t,U,Nt,pen,V", BH)
def test_bosehubbard_oracle_matches_reference(mpo_npz, name, L, N, t, U, Nt, pen, V):
    ws = mo.bosehubbard_hmpo(L, N, t, U, Nt, pen, V)
    for k in range(L):
        ref = mpo_npz[f"{name}_{k}"]
        assert ws[k].shape == ref.shape
        if name == "bh6":
            np.testing.assert_array_equal(ws[k], ref)
        else:  # the reference sums C * Z in its BLAS's order: last-bit differences
            np.testing.assert_allclose(ws[k], ref, rtol=0, atol=4.5e-16)


@pytest.mark.parametrize("name,L,N,t,U,Nt,pen,V", BH)
def test_bosehubbard_library_builder_matches_reference(dump_bin, mpo_npz, name, L, N, t, U, Nt, pen, V):
    ws = library_bh(dump_bin, L, N, t, U, Nt, pen, V)
    for k in range(L):
        ref = mpo_npz[f"{name}_{k}"]
        assert ws[k].shape == ref.shape
        if name == "bh6":
            np.testing.assert_array_equal(ws[k], ref)
        else:
            np.testing.assert_allclose(ws[k], ref, rtol=0, atol=4.5e-16)


def test_bosehubbard_mpo_is_the_hamiltonian():
    """-t sum (b+b + h.c.) + U/2 sum n(n-1) + V sum n + pen (sum n - Nt)^2,
    written out with Kronecker products, equals the contracted MPO."""
    L, N, t, U, Nt, pen, V = 4, 2, 0.8, 1.7, 3, 0.6, 0.35
    d = N + 1
    b = np.diag(np.sqrt(np.arange(1, d)), 1)   # annihilation
    n = np.diag(np.arange(d, dtype=float))
    eye = np.eye(d)

    def site(op, k):
        # basis index sum_k s_k d^k (the first site fastest, as mpo_dense)
        out = np.array([[1.0]])
        for j in reversed(range(L)):
            out = np.kron(out, op if j == k else eye)
        return out

    ntot = sum(site(n, k) for k in range(L))
    H = -t * sum(site(b.T, k) @ site(b, k + 1) + site(b, k) @ site(b.T, k + 1) for k in range(L - 1))
    H = H + sum(0.5 * U * site(n @ (n - eye), k) + V * site(n, k) for k in range(L))
    H = H + pen * (ntot - Nt * np.eye(d ** L)) @ (ntot - Nt * np.eye(d ** L))
    M = mo.mpo_dense(mo.bosehubbard_hmpo(L, N, t, U, Nt, pen, V))
    np.testing.assert_allclose(M, H, atol=1e-12)


def test_bosehubbard_ground_state_matches_reference(golden):
    """The oracle's sweep (the reference's algorithm) from the same seeded
    initial state as the reference run reaches its energy."""
    ops = mo.bosehubbard_hmpo(8, 2, 1.0, 2.0, 4, 1.0, 0.0)
    e = mo.find_ground_state(ops, 12, mo.random_mps(8, 3, 12, 6), convtol=1e-10)
    ref = golden["bosehubbard_L8_N2_D12_seed6_E0"]
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)
