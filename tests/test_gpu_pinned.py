"""GPU parity at the sizes that are timed, against the reference itself
(tests/golden/make_golden_large.py: the reference compiled from source with
the eigensolver shim, on the same seeded inputs, uploaded bit-exactly).

* the headline workload: Schwinger N=100, x=100, m/g=0.125 (mu=2.5), D=128,
  E0 from the seed-1 MPS and E1 from the seed-11 MPS, convtol 1e-10, in
  complex FP64 and in the mixed precision of the bench line;
* a request of the serving mix: Ising L=128, J=1, g=1, h=0.1, D=64, seed 7;
* the first 20 steps of a quench of the batched time-evolution workload:
  L=64, g=1.6490052627416842, h=0.1, dt=0.01, D<=64, <sigma_x> at the
  centre and the centre-bond entropy after every step.

Tolerances: |dE/E| <= 1e-10 for energies (the gap to 2e-10 |E0|), 1e-8
absolute for <sigma_x> and the entropy.
"""
import numpy as np
import pytest

from oracle import mps_oracle as mo

pytestmark = pytest.mark.gpu

MU = 2 * 0.125 * np.sqrt(100.0)
G_QUENCH = 1.6490052627416842


@pytest.mark.parametrize("precision", [0, 1])
def test_schwinger_N100_D128_E0_E1_gap(ctx, golden, precision):
    if "schwinger_N100_D128_seed11_E1" not in golden:
        pytest.skip("reference result not generated yet (tests/golden/make_golden_large.py)")
    E0r = golden["schwinger_N100_D128_seed1_E0"]
    E1r = golden["schwinger_N100_D128_seed11_E1"]
    H = ctx.mpo_schwinger(100, MU, 100.0)
    g = ctx.mps(mo.random_mps(100, 2, 128, 1).sites)
    x = ctx.mps(mo.random_mps(100, 2, 128, 11).sites)
    o = ctx.options(convtol=1e-10, precision=precision)
    e0, s0 = ctx.find_ground_state(H, 128, g, 0.0, o)
    e1, s1 = ctx.find_next_excited_state(H, 128, [g], x, 0.0, o)
    assert abs(e0 - E0r) <= 1e-10 * abs(E0r), (precision, e0, E0r)
    assert abs(e1 - E1r) <= 1e-10 * abs(E1r), (precision, e1, E1r)
    assert abs((e1 - e0) - (E1r - E0r)) <= 2e-10 * abs(E0r), (precision, e1 - e0, E1r - E0r)
    if precision == 1:
        assert s0["split_matvecs"] > 0 and s1["split_matvecs"] > 0


@pytest.mark.parametrize("precision", [0, 1])
def test_ising_L128_D64_request(ctx, golden, precision):
    ref = golden["ising_L128_D64_g1_h01_seed7_E0"]
    H = ctx.mpo_ising(128, 1.0, 1.0, 0.1)
    s = ctx.mps(mo.random_mps(128, 2, 64, 7).sites)
    e, _ = ctx.find_ground_state(H, 64, s, 0.0, ctx.options(convtol=1e-10, precision=precision))
    assert abs(e - ref) <= 1e-10 * abs(ref), (precision, e, ref)


def test_quench_L64_first_20_steps(ctx, golden):
    L, D = 64, 64
    U = ctx.mpo_ising_evolution(L, 1.0, G_QUENCH, 0.1, 0.01, False)
    H = ctx.mpo_ising(L, 1.0, G_QUENCH, 0.1)
    st = ctx.mps_product(L, 2, 1)
    o = ctx.options(convtol=1e-10)
    sx, ent, en = [], [], []
    for _ in range(20):
        aux = st.copy()
        ctx.optimize(U, aux, st, D, o)
        aux.free()
        sx.append(ctx.expectation_local(st, mo.SIGX)[L // 2])
        st.gauge("L")
        en.append(ctx.contract(st, H, st).real)
        ent.append(ctx.entropy(st, L // 2))
    np.testing.assert_allclose(sx, golden["quench_L64_D64_g1649_h01_dt001_sx_center"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(ent, golden["quench_L64_D64_g1649_h01_dt001_entropy_center"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(en, golden["quench_L64_D64_g1649_h01_dt001_energies"], rtol=1e-10, atol=0)
