"""CPU tests that pin the numpy oracle (oracle/mps_oracle.py) to the reference.

The golden fixtures in tests/golden were produced by the reference library
itself, compiled from source (oracle/Makefile), by tests/golden/make_golden.py.
Independent checks: exact diagonalisation and the free-fermion energy of the
open transverse-field Ising chain.
"""
import numpy as np
import pytest

from oracle import mps_oracle as mo

MU = 2 * 0.125 * np.sqrt(100.0)


def test_mpo_builders_bit_exact(mpo_npz):
    ops = {
        "ising6": mo.ising_hmpo(6, 1.0, 1.0, 0.3),
        "schwinger6": mo.schwinger_hmpo(6, 2.5, 100.0),
    }
    for name, lst in ops.items():
        for k in range(6):
            ref = mpo_npz[f"{name}_{k}"]
            assert ref.shape == lst[k].shape
            assert np.array_equal(ref, lst[k]), (name, k)
    for name, imag in [("uimag6", True), ("ureal6", False)]:
        u = mo.ising_umpo(6, 1.0, 1.0, 0.3, 0.01, imag)
        for k in range(6):
            ref = mpo_npz[f"{name}_{k}"]
            assert ref.shape == u[k].shape
            np.testing.assert_allclose(u[k], ref, rtol=0, atol=1e-15)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_kernels_match_reference(kernels_npz, tag):
    g = lambda n: kernels_npz[f"{tag}_{n}"]
    L, W, R, x = g("L"), g("W"), g("R"), g("x")
    y = mo.heff_matvec(L, W, R, x, 0.75)
    np.testing.assert_allclose(y, g("y_off075"), rtol=1e-13, atol=1e-12 * np.abs(y).max())
    yh = mo.heff_matvec_hermitian(L, W, R, x)
    np.testing.assert_allclose(yh, g("yherm"), rtol=1e-13, atol=1e-12 * np.abs(yh).max())
    eL = mo.env_left(g("TL"), g("ket"), W, g("bra"))
    np.testing.assert_allclose(eL, g("envL"), rtol=1e-13, atol=1e-12 * np.abs(eL).max())
    eR = mo.env_right(g("TR"), g("ket"), W, g("bra"))
    np.testing.assert_allclose(eR, g("envR"), rtol=1e-13, atol=1e-12 * np.abs(eR).max())
    # the dense effective Hamiltonian agrees with the matvec
    M = mo.heff_dense(L, W, R)
    np.testing.assert_allclose(M @ x + 0.75 * x, y, rtol=1e-12, atol=1e-11 * np.abs(y).max())


def test_bond_schedule_integers():
    assert mo.bond_schedule(20, 2, 20) == [1, 2, 4, 8, 16] + [20] * 11 + [16, 8, 4, 2, 1]
    assert mo.bond_schedule(6, 2, 128) == [1, 2, 4, 8, 4, 2, 1]
    m = mo.product_mps(6, 2, 8)
    mo.increase_bond_dimension(m, 8)  # no-op: bond already 8
    assert [a.shape for a in m.sites][0] == (2, 1, 8)
    m = mo.product_mps(6, 2, 1)
    mo.increase_bond_dimension(m, 8)
    assert [a.shape[2] for a in m.sites] == [2, 4, 8, 4, 2, 1]


def test_random_mps_is_seeded():
    a = mo.random_mps(8, 2, 4, 7)
    b = mo.random_mps(8, 2, 4, 7)
    c = mo.random_mps(8, 2, 4, 8)
    assert all(np.array_equal(x, y) for x, y in zip(a.sites, b.sites))
    assert not np.array_equal(a.sites[3], c.sites[3])
    z = np.concatenate([s.ravel() for s in mo.random_mps(40, 2, 16, 0).sites])
    assert abs(z.real.mean()) < 0.02 and abs(z.real.std() - 1) < 0.02


def test_mps_file_roundtrip(tmp_path):
    m = mo.random_mps(6, 2, 4, 3)
    m.normfact = 0.5
    fn = str(tmp_path / "m.mps")
    mo.write_mps(fn, m)
    r = mo.read_mps(fn)
    assert r.L == 6 and r.normfact == 0.5 and r.bond == 4
    assert all(np.array_equal(x, y) for x, y in zip(m.sites, r.sites))


@pytest.mark.parametrize("L", [6, 8])
def test_exact_diag_and_free_fermions(L):
    H = mo.mpo_dense(mo.ising_hmpo(L, 1.0, 1.0, 0.0))
    assert np.abs(H - H.conj().T).max() == 0
    e = np.linalg.eigvalsh(H)[0]
    assert abs(e - mo.tfim_open_energy(L, 1.0, 1.0)) < 1e-12 * abs(e)


def test_gs_ising_matches_reference(golden):
    m = mo.random_mps(10, 2, 8, 0)
    e = mo.find_ground_state(mo.ising_hmpo(10, 1, 1, 0), 8, m, convtol=1e-10)
    assert abs(e - golden["ising_L10_D8_seed0_E0"]) <= 1e-10 * abs(e)
    # D=8 at L=10 is close to exact
    assert abs(e - mo.tfim_open_energy(10, 1, 1)) < 1e-6


def test_gs_ising_field_matches_reference(golden):
    m = mo.random_mps(12, 2, 16, 3)
    e = mo.find_ground_state(mo.ising_hmpo(12, 1, 0.8, 0.1), 16, m, convtol=1e-10)
    assert abs(e - golden["ising_L12_D16_h01_seed3_E0"]) <= 1e-10 * abs(e)


def test_gs_schwinger_lanczos_branch_matches_reference(golden):
    # local dimension up to 2*24*24 = 1152 > 800: the PRIMME branch
    m = mo.random_mps(16, 2, 24, 1)
    e = mo.find_ground_state(mo.schwinger_hmpo(16, MU, 100.0), 24, m, convtol=1e-10)
    assert abs(e - golden["schwinger_N16_D24_seed1_E0"]) <= 1e-10 * abs(e)


def test_excited_state_matches_reference(golden):
    ops = mo.ising_hmpo(10, 1, 1, 0)
    g = mo.random_mps(10, 2, 16, 1)
    x = mo.random_mps(10, 2, 16, 11)
    e0 = mo.find_ground_state(ops, 16, g, convtol=1e-10)
    e1 = mo.find_next_excited_state(ops, 16, [g], x, convtol=1e-10)
    assert abs(e0 - golden["ising_L10_D16_exc_E0"]) <= 1e-10 * abs(e0)
    assert abs(e1 - golden["ising_L10_D16_exc_E1"]) <= 1e-10 * abs(e1)
    w = np.linalg.eigvalsh(mo.mpo_dense(ops))
    assert abs(e1 - w[1]) < 1e-8 * abs(w[1])


def test_imaginary_time_matches_reference(golden):
    L, D = 10, 6
    ops = mo.ising_hmpo(L, 1, 1, 0)
    U = mo.ising_umpo(L, 1, 1, 0, 0.05, True)
    st = mo.product_mps(L, 2, D)
    es = []
    for _ in range(20):
        aux = st.copy()
        mo.optimize(U, aux, st, D, convtol=1e-10)
        mo.gauge_cond_all(st, "R", True)
        es.append(mo.contract_op(st, ops, st).real)
    ref = np.array(golden["ising_L10_D6_imag_dt005_energies"])
    np.testing.assert_allclose(es, ref, rtol=1e-10, atol=0)


def test_real_time_quench_matches_reference(golden):
    L, D = 8, 8
    ops = mo.ising_hmpo(L, 1, 1.2, 0.1)
    U = mo.ising_umpo(L, 1, 1.2, 0.1, 0.05, False)
    st = mo.product_mps(L, 2, 1)
    sx, en, ent = [], [], []
    for _ in range(10):
        aux = st.copy()
        mo.optimize(U, aux, st, D, convtol=1e-10)
        sx.append(mo.expectation_values(st, mo.SIGX)[L // 2])
        mo.gauge_cond_all(st, "L", True)
        en.append(mo.contract_op(st, ops, st).real)
        ent.append(mo.entropy(st, L // 2))
    np.testing.assert_allclose(sx, golden["ising_L8_D8_quench_sx_center"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(en, golden["ising_L8_D8_quench_energies"], rtol=1e-10, atol=0)
    np.testing.assert_allclose(ent, golden["ising_L8_D8_quench_entropy"], rtol=0, atol=1e-8)


def test_qr_lq_conventions_match_lapack():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((12, 5)) + 1j * rng.standard_normal((12, 5))
    Q, R = mo.qr_reduced(A)
    np.testing.assert_allclose(Q @ R, A, atol=1e-13)
    Lm, Q2 = mo.lq_reduced(A.T.copy())
    np.testing.assert_allclose(Lm @ Q2, A.T, atol=1e-13)
    np.testing.assert_allclose(Q2 @ Q2.conj().T, np.eye(5), atol=1e-13)


def test_random_state_is_normalised_isometry_chain():
    m = mo.random_state(10, 2, 6, 3)
    assert abs(mo.contract_overlap(m, m).real - 1.0) < 1e-12
    for a in m.sites:
        d, Dl, Dr = a.shape
        M = a.reshape(d * Dl, Dr, order="F")
        assert np.abs(M.conj().T @ M - np.eye(Dr)).max() < 1e-13


def test_truncation_matches_reference(trunc_npz):
    t = mo.truncate_mps(mo.random_mps(10, 2, 16, 21), 5)
    np.testing.assert_array_equal(np.array([a.shape for a in t.sites]), trunc_npz["trunc_L10_D16_seed21_to5_dims"])
    ref = trunc_npz["trunc_L10_D16_seed21_to5_vec"]
    assert np.abs(mo.mps_to_vector(t) - ref).max() < 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("cut", [0, 4])
@pytest.mark.parametrize("dagger", [0, 1])
@pytest.mark.parametrize("direction", ["L", "R"])
def test_apply_mpo_matches_reference(trunc_npz, cut, dagger, direction):
    U = mo.ising_umpo(8, 1.0, 1.1, 0.2, 0.05, False)
    t = mo.apply_mpo(U, mo.random_mps(8, 2, 6, 5), cut, bool(dagger), direction)
    tag = f"apply_L8_D6_seed5_ureal005_cut{cut}_dag{dagger}_{direction}"
    np.testing.assert_array_equal(np.array([a.shape for a in t.sites]), trunc_npz[tag + "_dims"])
    ref = trunc_npz[tag + "_vec"]
    assert np.abs(mo.mps_to_vector(t) - ref).max() < 1e-12 * np.abs(ref).max()


def test_gs_prologue_truncates_large_initial_bond(golden):
    m = mo.random_mps(12, 2, 16, 4)
    e = mo.find_ground_state(mo.ising_hmpo(12, 1, 1, 0), 6, m, convtol=1e-10)
    ref = golden["ising_L12_init16_D6_seed4_E0"]
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)


def test_contract2_matches_reference(golden):
    m = mo.random_mps(8, 2, 6, 7)
    for key, H in (("contract2_ising_L8_D6_seed7", mo.ising_hmpo(8, 1, 1.1, 0.2)),
                   ("contract2_schwinger_N8_D6_seed7", mo.schwinger_hmpo(8, 2.5, 100.0))):
        v = mo.contract2(H, m)
        assert abs(v.real - golden[key]) < 1e-12 * abs(golden[key]), (key, v)


def test_optimize_error_matches_reference(golden):
    orig = mo.random_state(8, 2, 6, 9)
    init = orig.copy()
    U = mo.ising_umpo(8, 1.0, 1.1, 0.2, 0.05, False)
    mo.optimize(U, orig, init, 6, convtol=1e-10)
    errN, errT = mo.optimize_error(U, orig, init)
    rN, rT, rnf = golden["opterr_ising_L8_D6_state9_ureal005"]
    assert abs(errN - rN) < 1e-11 and abs(errT - rT) < 1e-12 and abs(init.normfact - rnf) < 1e-12


def test_two_site_oracle_exact_tfim():
    L, g = 8, 1.3
    m = mo.product_mps(L, 2, 1)
    e, dw = mo.find_ground_state_two_site(mo.ising_hmpo(L, 1, g, 0), 16, m, convtol=1e-10)
    exact = mo.tfim_open_energy(L, 1, g)
    assert abs(e - exact) <= 1e-10 * abs(exact) and dw == 0.0


def test_imaginary_time_L20_config(golden):
    L, D = 20, 20
    H, U = mo.ising_hmpo(L, 1, 1, 0), mo.ising_umpo(L, 1, 1, 0, 0.01, True)
    st = mo.product_mps(L, 2, D)
    es = []
    for _ in range(200):
        aux = st.copy()
        mo.optimize(U, aux, st, D, convtol=1e-10)
        mo.gauge_cond_all(st, "R", True)
        es.append(mo.contract_op(st, H, st).real)
    np.testing.assert_allclose(es, golden["ising_L20_D20_imag_dt001_M200_energies"], rtol=1e-10, atol=0)


def test_heisenberg_mpo_bit_exact(mpo_npz):
    ops = mo.heisenberg_hmpo(6, 1, 0.8, 1.2, 0.3, 0.1, 0.5, 0.7)
    for k in range(6):
        np.testing.assert_array_equal(ops[k], mpo_npz[f"heis6_{k}"])


def test_heisenberg_gs_matches_reference(golden):
    e = mo.find_ground_state(mo.heisenberg_hmpo(10, 1, 1, 1), 16, mo.random_mps(10, 2, 16, 0), convtol=1e-10)
    ref = golden["heisenberg_L10_D16_seed0_E0"]
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)
