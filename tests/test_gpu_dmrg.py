"""GPU parity of the DMRG sweep (Contractor::findGroundState and friends)
through the C ABI, on the same seeded initial states as the reference runs
that produced tests/golden/golden.json.

Tolerance: |dE/E| <= 1e-10 (the energy bound of the target), observables
<= 1e-8.
"""
import numpy as np
import pytest

from oracle import mps_oracle as mo

pytestmark = pytest.mark.gpu

MU = 2 * 0.125 * np.sqrt(100.0)


def solve_gs(ctx, ops, mps, D, convtol=1e-10):
    m = ctx.mpo(ops)
    s = ctx.mps(mps.sites, mps.normfact)
    e, st = ctx.find_ground_state(m, D, s, 0.0, ctx.options(convtol=convtol))
    return e, st, m, s


def test_gs_ising_L10(ctx, golden):
    e, st, m, s = solve_gs(ctx, mo.ising_hmpo(10, 1, 1, 0), mo.random_mps(10, 2, 8, 0), 8)
    ref = golden["ising_L10_D8_seed0_E0"]
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)
    assert st["matvecs"] > 0 and st["rounds"] >= 2
    # the returned state is the ground state: <H> agrees, norm 1
    assert abs(ctx.contract(s, m, s).real - e) < 1e-9 * abs(e)
    assert abs(ctx.contract(s, None, s).real - 1.0) < 1e-12


def test_gs_ising_L20_D20_config(ctx, golden):
    e, st, m, s = solve_gs(ctx, mo.ising_hmpo(20, 1, 1, 0), mo.random_mps(20, 2, 20, 0), 20)
    ref = golden["ising_L20_D20_seed0_E0"]
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)


def test_gs_ising_field(ctx, golden):
    e, *_ = solve_gs(ctx, mo.ising_hmpo(12, 1, 0.8, 0.1), mo.random_mps(12, 2, 16, 3), 16)
    ref = golden["ising_L12_D16_h01_seed3_E0"]
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)


def test_gs_schwinger(ctx, golden):
    e, *_ = solve_gs(ctx, mo.schwinger_hmpo(16, MU, 100.0), mo.random_mps(16, 2, 24, 1), 24)
    ref = golden["schwinger_N16_D24_seed1_E0"]
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)


def test_gs_free_fermion_energy(ctx):
    L = 16
    e, *_ = solve_gs(ctx, mo.ising_hmpo(L, 1, 0.7, 0), mo.random_mps(L, 2, 32, 9), 32)
    exact = mo.tfim_open_energy(L, 1, 0.7)
    assert abs(e - exact) < 1e-9 * abs(exact)


def test_gauge_and_download_roundtrip(ctx):
    m = mo.random_mps(8, 2, 6, 4)
    s = ctx.mps(m.sites)
    n0 = ctx.contract(s, None, s).real
    s.gauge("R")
    sites, nf = s.download()
    r = mo.MPS([np.asarray(a) for a in sites], nf)
    assert abs(mo.contract_overlap(r, r).real - 1.0) < 1e-12
    # left-isometries after the right sweep (except the last site)
    for a in sites[:-1]:
        d, Dl, Dr = a.shape
        M = a.reshape(d * Dl, Dr, order="F")
        assert np.abs(M.conj().T @ M - np.eye(Dr)).max() < 1e-13
    assert n0 > 0


def test_device_random_state_matches_generator(ctx):
    s = ctx.mps_random(10, 2, 8, 77)
    sites, _ = s.download()
    ref = mo.random_mps(10, 2, 8, 77)
    for a, b in zip(sites, ref.sites):
        assert a.shape == b.shape
        assert np.abs(a - b).max() < 1e-13 * np.abs(b).max()


def test_errors_are_status_codes(ctx):
    from mpsdyn_b200 import capi
    ops = ctx.mpo(mo.ising_hmpo(6, 1, 1, 0))
    s = ctx.mps(mo.random_mps(8, 2, 4, 0).sites)  # wrong length
    with pytest.raises(capi.MpsgpuError) as ei:
        ctx.find_ground_state(ops, 4, s)
    assert ei.value.status == 1


def test_excited_state_matches_reference(ctx, golden):
    ops = ctx.mpo(mo.ising_hmpo(10, 1, 1, 0))
    g = ctx.mps(mo.random_mps(10, 2, 16, 1).sites)
    x = ctx.mps(mo.random_mps(10, 2, 16, 11).sites)
    o = ctx.options(convtol=1e-10)
    e0, _ = ctx.find_ground_state(ops, 16, g, 0.0, o)
    e1, st = ctx.find_next_excited_state(ops, 16, [g], x, 0.0, o)
    r0, r1 = golden["ising_L10_D16_exc_E0"], golden["ising_L10_D16_exc_E1"]
    assert abs(e0 - r0) <= 1e-10 * abs(r0)
    assert abs(e1 - r1) <= 1e-10 * abs(r1), (e1, r1)
    # orthogonal to the ground state
    assert abs(ctx.contract(x, None, g)) < 1e-6


def test_imaginary_time_matches_reference(ctx, golden):
    L, D = 10, 6
    H = ctx.mpo(mo.ising_hmpo(L, 1, 1, 0))
    U = ctx.mpo(mo.ising_umpo(L, 1, 1, 0, 0.05, True))
    st = ctx.mps_product(L, 2, D)
    o = ctx.options(convtol=1e-10)
    es = []
    for _ in range(20):
        aux = st.copy()
        ctx.optimize(U, aux, st, D, o)
        aux.free()
        st.gauge("R")
        es.append(ctx.contract(st, H, st).real)
    np.testing.assert_allclose(es, golden["ising_L10_D6_imag_dt005_energies"], rtol=1e-10, atol=0)


def test_real_time_quench_observables(ctx, golden):
    L, D = 8, 8
    H = ctx.mpo(mo.ising_hmpo(L, 1, 1.2, 0.1))
    U = ctx.mpo(mo.ising_umpo(L, 1, 1.2, 0.1, 0.05, False))
    st = ctx.mps(mo.product_mps(L, 2, 1).sites)
    o = ctx.options(convtol=1e-10)
    sx, en = [], []
    for _ in range(10):
        aux = st.copy()
        ctx.optimize(U, aux, st, D, o)
        aux.free()
        sx.append(ctx.expectation_local(st, mo.SIGX)[L // 2])
        st.gauge("L")
        en.append(ctx.contract(st, H, st).real)
    np.testing.assert_allclose(sx, golden["ising_L8_D8_quench_sx_center"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(en, golden["ising_L8_D8_quench_energies"], rtol=1e-10, atol=0)


@pytest.mark.parametrize("pos", [0, 3, 5, 9])
def test_schmidt_values_and_entropy_vs_oracle(ctx, pos):
    m = mo.random_mps(9, 2, 6, 33)
    s = ctx.mps(m.sites)
    lam = ctx.schmidt_values(s, pos)
    ref = mo.schmidt_values(m, pos)
    assert lam.shape == ref.shape
    np.testing.assert_allclose(lam, ref, rtol=0, atol=1e-12)
    assert abs(ctx.entropy(s, pos) - mo.entropy(m, pos)) < 1e-10


def test_quench_entropy_matches_reference(ctx, golden):
    L, D = 8, 8
    U = ctx.mpo(mo.ising_umpo(L, 1, 1.2, 0.1, 0.05, False))
    st = ctx.mps(mo.product_mps(L, 2, 1).sites)
    o = ctx.options(convtol=1e-10)
    ent = []
    for _ in range(10):
        aux = st.copy()
        ctx.optimize(U, aux, st, D, o)
        aux.free()
        st.gauge("L")
        ent.append(ctx.entropy(st, L // 2))
    np.testing.assert_allclose(ent, golden["ising_L8_D8_quench_entropy"], rtol=0, atol=1e-8)


def test_zero_padded_gauge_matches_oracle(ctx):
    # a product state zero-padded to D=64 (what optimize sees for a D=1 start)
    m = mo.product_mps(16, 2, 1)
    mo.increase_bond_dimension(m, 64)
    s = ctx.mps(m.sites)
    ref = m.copy()
    for d_ in ("R", "L"):
        s.gauge(d_)
        mo.gauge_cond_all(ref, d_, True)
        sites, _ = s.download()
        for k, (a, b) in enumerate(zip(sites, ref.sites)):
            assert a.shape == b.shape, (d_, k)
            assert np.all(np.isfinite(a)), (d_, k)
            assert np.abs(a - b).max() < 1e-12, (d_, k, np.abs(a - b).max())


def test_quench_from_product_state_D64_vs_oracle(ctx):
    # the optimised sites are rank-deficient: their LQ meets trailing columns
    # with entries far below 1e-154, whose plain squares underflow
    L, D = 16, 64
    U = ctx.mpo(mo.ising_umpo(L, 1, 1.0, 0.1, 0.01, False))
    st = ctx.mps(mo.product_mps(L, 2, 1).sites)
    ref = mo.product_mps(L, 2, 1)
    Ur = mo.ising_umpo(L, 1, 1.0, 0.1, 0.01, False)
    o = ctx.options(convtol=1e-10)
    for _ in range(2):
        aux = st.copy()
        ctx.optimize(U, aux, st, D, o)
        aux.free()
        raux = ref.copy()
        mo.optimize(Ur, raux, ref, D, convtol=1e-10)
        assert abs(ctx.expectation_local(st, mo.SIGX)[L // 2] - mo.expectation_values(ref, mo.SIGX)[L // 2]) < 1e-8


def test_expectation_values_vs_oracle(ctx):
    m = mo.random_mps(9, 2, 6, 21)
    s = ctx.mps(m.sites)
    for op in (mo.SIGX, mo.SIGZ, mo.SIGY):
        np.testing.assert_allclose(ctx.expectation_local(s, op), mo.expectation_values(m, op), rtol=0, atol=1e-12)


def test_random_state_matches_oracle(ctx):
    s = ctx.mps_random_state(12, 2, 8, 5)
    sites, nf = s.download()
    ref = mo.random_state(12, 2, 8, 5)
    assert nf == 1.0
    for a, b in zip(sites, ref.sites):
        assert a.shape == b.shape
        assert np.abs(a - b).max() < 1e-12
    assert abs(ctx.contract(s, None, s).real - 1.0) < 1e-12


def test_gs_long_chain_from_random_state(ctx):
    # L = 240: the raw Gaussian chain would overflow (norm ~ (d D)^(L/2));
    # the gauged random state does not.  Gapped TFIM, exact energy by free fermions.
    L, D, g = 240, 16, 2.0
    m = ctx.mpo_ising(L, 1.0, g, 0.0)
    s = ctx.mps_random_state(L, 2, D, 3)
    e, st = ctx.find_ground_state(m, D, s, 0.0, ctx.options(convtol=1e-10))
    exact = mo.tfim_open_energy(L, 1.0, g)
    assert abs(e - exact) < 1e-9 * abs(exact), (e, exact)


@pytest.mark.parametrize("krylov", [6, 16])
def test_gs_with_small_krylov_space_restarts(ctx, golden, krylov):
    # a short Krylov space forces many thick restarts per site
    ops = ctx.mpo(mo.ising_hmpo(20, 1, 1, 0))
    s = ctx.mps(mo.random_mps(20, 2, 20, 0).sites)
    e, st = ctx.find_ground_state(ops, 20, s, 0.0, ctx.options(convtol=1e-10, max_krylov=krylov))
    ref = golden["ising_L20_D20_seed0_E0"]
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)


def test_contract2_matches_reference(ctx, golden):
    s = ctx.mps(mo.random_mps(8, 2, 6, 7).sites)
    for key, H in (("contract2_ising_L8_D6_seed7", mo.ising_hmpo(8, 1, 1.1, 0.2)),
                   ("contract2_schwinger_N8_D6_seed7", mo.schwinger_hmpo(8, 2.5, 100.0))):
        v = ctx.contract2(ctx.mpo(H), s)
        assert abs(v.real - golden[key]) < 1e-12 * abs(golden[key]), (key, v)


def test_optimize_error_matches_reference(ctx, golden):
    orig = ctx.mps_random_state(8, 2, 6, 9)
    init = orig.copy()
    U = ctx.mpo(mo.ising_umpo(8, 1.0, 1.1, 0.2, 0.05, False))
    errN, errT, _ = ctx.optimize(U, orig, init, 6, ctx.options(convtol=1e-10), want_err=True)
    rN, rT, rnf = golden["opterr_ising_L8_D6_state9_ureal005"]
    assert abs(errN - rN) < 1e-11 and abs(errT - rT) < 1e-12
    assert abs(init.info()[2] - rnf) < 1e-12


def test_imaginary_time_L20_config_matches_reference(ctx, golden):
    # testIsing.cpp's imaginary-time phase at L = 20, D = 20: 200 steps of
    # delta = 0.01 from MPS(L, D, d)
    L, D = 20, 20
    H = ctx.mpo(mo.ising_hmpo(L, 1, 1, 0))
    U = ctx.mpo(mo.ising_umpo(L, 1, 1, 0, 0.01, True))
    st = ctx.mps_product(L, 2, D)
    o = ctx.options(convtol=1e-10)
    es = []
    for _ in range(200):
        aux = st.copy()
        ctx.optimize(U, aux, st, D, o)
        aux.free()
        st.gauge("R")
        es.append(ctx.contract(st, H, st).real)
    np.testing.assert_allclose(es, golden["ising_L20_D20_imag_dt001_M200_energies"], rtol=1e-10, atol=0)
