"""GPU parity of the CUDA kernels against the oracle, through the C ABI.

Tolerances: complex FP64 throughout, so products agree with the oracle to a
few ulps of the largest term (relative error <= 1e-13 of max |y|).
"""
import numpy as np
import pytest

from oracle import mps_oracle as mo

pytestmark = pytest.mark.gpu


def rand_c(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_matvec_and_env_vs_reference_fixture(ctx, kernels_npz, tag):
    g = lambda n: kernels_npz[f"{tag}_{n}"]
    L, W, R, x = g("L"), g("W"), g("R"), g("x")
    assert rel(ctx.heff_matvec(L, W, R, x, 0.75), g("y_off075")) < 1e-13
    assert rel(ctx.heff_matvec(L, W, R, x, hermitian=True), g("yherm")) < 1e-13
    assert rel(ctx.env_left(g("TL"), g("ket"), W, g("bra")), g("envL")) < 1e-13
    assert rel(ctx.env_right(g("TR"), g("ket"), W, g("bra")), g("envR")) < 1e-13


@pytest.mark.parametrize("D,w,d", [(8, 3, 2), (20, 3, 2), (64, 5, 2), (128, 5, 2), (33, 4, 3)])
def test_matvec_random_shapes(ctx, D, w, d):
    rng = np.random.default_rng(D * 10 + w)
    Dl, Dr = D, D + 3
    L = rand_c(rng, (Dl, w, Dl))
    W = rand_c(rng, (d, w, d, w))
    R = rand_c(rng, (Dr, w, Dr))
    x = rand_c(rng, (d * Dl * Dr,))
    y = ctx.heff_matvec(L, W, R, x, 0.3)
    assert rel(y, mo.heff_matvec(L, W, R, x, 0.3)) < 1e-13
    T = rand_c(rng, (Dl, w, Dl))
    ket = rand_c(rng, (d, Dl, Dr))
    bra = rand_c(rng, (d, Dl, Dr))
    assert rel(ctx.env_left(T, ket, W, bra), mo.env_left(T, ket, W, bra)) < 1e-13
    T2 = rand_c(rng, (Dr, w, Dr))
    assert rel(ctx.env_right(T2, ket, W, bra), mo.env_right(T2, ket, W, bra)) < 1e-13


def test_matvec_rectangular_environments(ctx):
    rng = np.random.default_rng(5)
    L = rand_c(rng, (7, 3, 5))
    W = rand_c(rng, (2, 3, 2, 3))
    R = rand_c(rng, (6, 3, 9))
    x = rand_c(rng, (2 * 5 * 9,))
    assert rel(ctx.heff_matvec(L, W, R, x), mo.heff_matvec(L, W, R, x)) < 1e-13


@pytest.mark.parametrize("m,n", [(2, 1), (4, 2), (40, 20), (256, 128), (200, 256), (512, 256), (17, 17), (3, 9)])
def test_qr_matches_lapack(ctx, m, n):
    rng = np.random.default_rng(m + 7 * n)
    A = rand_c(rng, (m, n))
    Q, R = ctx.qr(A)
    Qn, Rn = np.linalg.qr(A, mode="reduced")  # LAPACK zgeqrf/zungqr
    K = min(m, n)
    assert Q.shape == (m, K) and R.shape == (K, n)
    scale = np.abs(A).max()
    assert np.abs(Q @ R - A).max() < 1e-13 * scale * max(m, n) ** 0.5
    assert np.abs(Q.conj().T @ Q - np.eye(K)).max() < 1e-13 * max(m, n) ** 0.5
    assert np.abs(np.tril(R, -1)).max() == 0
    # same Householder conventions as LAPACK: same factors, not only the same product
    assert rel(R, Rn) < 1e-11
    assert rel(Q, Qn) < 1e-11


def test_qr_zero_padded_matches_lapack(ctx):
    # rank-deficient, zero-padded site as MPS(L, D, d) produces them
    A = np.zeros((8, 6), dtype=complex)
    A[0, 0] = 1.0
    A[3, 1] = 0.5 - 0.25j
    Q, R = ctx.qr(A)
    Qn, Rn = np.linalg.qr(A, mode="reduced")
    assert rel(Q, Qn) < 1e-14 and rel(R, Rn) < 1e-14


@pytest.mark.parametrize("scale", [1e-160, 1e150])
def test_qr_tiny_and_huge_columns_match_lapack(ctx, scale):
    # trailing columns far below (or above) the range whose squares are
    # representable: the reflectors are computed from rescaled columns, as
    # zlarfg does, so the factors still equal LAPACK's
    rng = np.random.default_rng(3)
    A = rand_c(rng, (64, 32))
    A[:, 20:] *= scale
    Q, R = ctx.qr(A)
    Qn, Rn = np.linalg.qr(A, mode="reduced")
    assert rel(Q, Qn) < 1e-11 and rel(R, Rn) < 1e-11
    assert np.abs(Q.conj().T @ Q - np.eye(32)).max() < 1e-13


def test_qr_tiny_pivots_and_signed_zero_match_lapack(ctx):
    # a column that is exactly zero below a tiny complex diagonal entry (its
    # squared modulus underflows), and a diagonal entry with real part -0.0
    # (LAPACK's sign(., -0.0) is negative)
    A = np.zeros((6, 3), dtype=complex)
    A[0, 0] = 1.0
    A[1, 1] = 1e-170 + 2e-170j
    A[2, 2] = complex(-0.0, -3e-200)
    A[4, 2] = 1e-201
    Q, R = ctx.qr(A)
    Qn, Rn = np.linalg.qr(A, mode="reduced")
    assert np.all(np.isfinite(Q)) and np.all(np.isfinite(R))
    assert rel(Q, Qn) < 1e-12
    for i in range(3):
        assert abs(R[i, i] - Rn[i, i]) <= 1e-12 * abs(Rn[i, i])


def test_qr_padded_site_256x128_matches_lapack(ctx):
    # a D = 128 site grown from bond dimension 40: the other columns are zero
    rng = np.random.default_rng(8)
    A = np.zeros((256, 128), dtype=complex)
    A[:80, :40] = rand_c(rng, (80, 40))
    Q, R = ctx.qr(A)
    Qn, Rn = np.linalg.qr(A, mode="reduced")
    assert rel(Q, Qn) < 1e-11 and rel(R, Rn) < 1e-11


@pytest.mark.parametrize("m,n", [(6, 20), (20, 6), (128, 256)])
def test_lq_matches_lapack(ctx, m, n):
    rng = np.random.default_rng(m * n)
    A = rand_c(rng, (m, n))
    Lm, Q = ctx.lq(A)
    Lr, Qr = mo.lq_reduced(A)
    assert np.abs(Lm @ Q - A).max() < 1e-13 * np.abs(A).max() * max(m, n) ** 0.5
    assert rel(Lm, Lr) < 1e-11 and rel(Q, Qr) < 1e-11


def test_gemm_autotuner_same_energy_on_and_off(ctx):
    """The GEMM autotuner only changes launch configurations: the sweep
    reaches the same energy with it off and on, and it records the shapes
    it tuned."""
    from mpsdyn_b200 import capi
    from oracle import mps_oracle as mo
    H = mo.ising_hmpo(12, 1, 0.9, 0.1)
    m = ctx.mpo(H)
    o = ctx.options(convtol=1e-10)
    energies = []
    try:
        for on in (False, True):
            capi.set_autotune(on)
            s = ctx.mps(mo.random_mps(12, 2, 16, 21).sites)
            e, _ = ctx.find_ground_state(m, 16, s, 0.0, o)
            energies.append(e)
    finally:
        capi.set_autotune(True)
    assert abs(energies[0] - energies[1]) <= 1e-10 * abs(energies[0])
    assert capi.autotune_entries() > 0
