"""Host-side pieces of the device Lanczos (mpsdyn_b200/csrc/tridiag.h),
compiled with g++ and checked against numpy: the tridiagonal eigenvalues by
bisection, and the thick restart (Wu & Simon 2000) that compresses an m-step
factorisation H V = V T + f e_m^T to about m/2 vectors in tridiagonal form."""
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def irl_bin(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("irl") / "irl_check"
    subprocess.run(["g++", "-O2", "-std=c++17", "-o", str(out), os.path.join(HERE, "native", "irl_check.cpp")],
                   check=True)
    return str(out)


def run(irl_bin, a, b, keep, fnorm):
    m = len(a)
    inp = (f"{m} {keep} {float(fnorm)!r}\n" + " ".join(repr(float(x)) for x in a) + "\n"
           + " ".join(repr(float(x)) for x in b) + "\n")
    lines = subprocess.run([irl_bin], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    r = int(lines[0])
    ap = np.array(lines[1].split(), float)
    bp = np.array(lines[2].split(), float)
    G = np.array(lines[3].split(), float).reshape(r, m).T
    ev = np.array(lines[4].split(), float)
    return r, ap, bp, G, ev


def tridiag(a, b):
    return np.diag(a) + np.diag(b[: len(a) - 1], 1) + np.diag(b[: len(a) - 1], -1)


def lanczos_matrix(rng, m, spectrum):
    """T_m and the residual norms of m reorthogonalised Lanczos steps on
    diag(spectrum)."""
    n = len(spectrum)
    v = rng.standard_normal(n)
    V = [v / np.linalg.norm(v)]
    a, b = [], []
    for j in range(m):
        w = spectrum * V[j]
        for _ in range(2):
            for q in V:
                w = w - (q @ w) * q
        a.append(float(V[j] @ (spectrum * V[j])))
        b.append(float(np.linalg.norm(w)))
        V.append(w / b[-1])
    return np.array(a), np.array(b)


CASES = [
    ("random", 12, 6, 0), ("random", 64, 32, 1), ("random", 9, 1, 2), ("random", 40, 20, 3),
    ("lanczos", 64, 32, 4), ("lanczos_cluster", 64, 32, 5), ("lanczos_degenerate", 48, 24, 6),
]


@pytest.mark.parametrize("kind,m,keep,seed", CASES)
def test_thick_restart_compression(irl_bin, kind, m, keep, seed):
    rng = np.random.default_rng(seed)
    if kind == "random":
        a = rng.standard_normal(m) * 3
        b = np.abs(rng.standard_normal(m)) + 0.1
    else:
        spec = np.sort(rng.uniform(-50, 50, 2000))
        if kind == "lanczos_cluster":
            spec[:3] = [-60.0, -60.0 + 1e-7, -60.0 + 3e-7]
        if kind == "lanczos_degenerate":
            spec[:2] = [-70.0, -70.0]
        a, b = lanczos_matrix(rng, m, spec)
    fnorm = b[m - 1]
    T = tridiag(a, b)
    r, ap, bp, G, ev = run(irl_bin, a, b, keep, fnorm)
    assert 1 <= r <= keep
    # orthonormal G; G^T T G is the compressed tridiagonal
    assert np.abs(G.T @ G - np.eye(r)).max() < 1e-12
    assert np.abs(G.T @ T @ G - tridiag(ap, bp)).max() < 1e-11 * np.abs(T).max()
    # only the last kept vector couples to f: |f| e_m^T G = |s| e_r^T
    cpl = fnorm * G[m - 1, :]
    assert np.abs(cpl[:-1]).max(initial=0.0) < 1e-11 * max(fnorm, 1.0)
    assert abs(abs(cpl[-1]) - bp[r - 1]) < 1e-11 * max(fnorm, 1.0)
    # the lowest Ritz value of T survives the restart
    lam0 = np.linalg.eigvalsh(T)[0]
    assert abs(np.linalg.eigvalsh(tridiag(ap, bp))[0] - lam0) < 1e-10 * np.abs(T).max()
    # bisection agrees with numpy on the compressed matrix
    assert np.abs(ev - np.linalg.eigvalsh(tridiag(ap, bp))).max() < 1e-12 * np.abs(T).max()


def _thick_restart_lanczos(irl_bin, H, m, tol=1e-12, max_restarts=60, seed=0):
    """The device loop of engine.cu (lanczos_lowest) in numpy, with the
    compiled compression: returns (lowest eigenvalue or None, matvecs)."""
    N = H.shape[0]
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    V = np.zeros((N, m + 1), complex)
    V[:, 0] = x / np.linalg.norm(x)
    a, b, j0, keep, total = [], [], 0, max(1, m // 2), 0
    for _ in range(max_restarts):
        for j in range(j0, m):
            w = H @ V[:, j]
            total += 1
            h1 = V[:, : j + 1].conj().T @ w
            w -= V[:, : j + 1] @ h1
            h2 = V[:, : j + 1].conj().T @ w
            w -= V[:, : j + 1] @ h2
            a.append((h1[j] + h2[j]).real)
            b.append(np.linalg.norm(w))
            ev, Y = np.linalg.eigh(tridiag(np.array(a), np.array(b)))
            if b[-1] * abs(Y[-1, 0]) <= tol * np.abs(ev).max():
                return ev[0], total
            if j + 1 < m:
                V[:, j + 1] = w / b[-1]
        r, ap, bp, G, _ = run(irl_bin, a, b, keep, b[m - 1])
        V[:, :r] = V[:, :m] @ G
        V[:, r] = w / np.linalg.norm(w)
        a, b, j0 = list(ap), list(bp), r
    return None, total


@pytest.mark.parametrize("m", [12, 24])
def test_thick_restart_lanczos_converges(irl_bin, m):
    rng = np.random.default_rng(1)
    N = 300
    A = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    H = (A + A.conj().T) / 2
    lam = np.linalg.eigvalsh(H)[0]
    e, total = _thick_restart_lanczos(irl_bin, H, m)
    assert e is not None and abs(e - lam) < 1e-10 * abs(lam), (e, lam, total)
