"""Mixed-precision sweeps (options.precision = 1): split-precision products
on the tensor cores until the half-sweep energy settles, FP64 to
convergence.  The energies must meet the same bound as the FP64 path,
|dE/E| <= 1e-10 against the reference's runs (tests/golden), and the
split phase must have run."""
import numpy as np
import pytest

from oracle import mps_oracle as mo

pytestmark = pytest.mark.gpu

MU = 2 * 0.125 * np.sqrt(100.0)
TOL = 1e-10


def mixed(ctx, **kw):
    return ctx.options(convtol=1e-10, precision=1, **kw)


@pytest.mark.parametrize("key,build,mps", [
    ("ising_L20_D20_seed0_E0", lambda: mo.ising_hmpo(20, 1, 1, 0), lambda: mo.random_mps(20, 2, 20, 0)),
    ("ising_L12_D16_h01_seed3_E0", lambda: mo.ising_hmpo(12, 1, 0.8, 0.1), lambda: mo.random_mps(12, 2, 16, 3)),
    ("schwinger_N16_D24_seed1_E0", lambda: mo.schwinger_hmpo(16, MU, 100.0), lambda: mo.random_mps(16, 2, 24, 1)),
])
def test_mixed_gs_matches_reference(ctx, golden, key, build, mps):
    m = ctx.mpo(build())
    st0 = mps()
    s = ctx.mps(st0.sites, st0.normfact)
    D = max(max(a.shape[1], a.shape[2]) for a in st0.sites)
    e, st = ctx.find_ground_state(m, D, s, 0.0, mixed(ctx))
    ref = golden[key]
    assert abs(e - ref) <= TOL * abs(ref), (e, ref)
    assert st["split_rounds"] >= 1 and st["split_matvecs"] > 0, st
    assert st["split_matvecs"] < st["matvecs"]  # the FP64 phase ran too
    assert abs(ctx.contract(s, m, s).real - e) < 1e-9 * abs(e)


def test_mixed_heisenberg_with_fields(ctx, golden):
    ops = ctx.mpo_heisenberg(12, 1, 0.7, 1.3, 0.2, 0.1, 0.4)
    s = ctx.mps(mo.random_mps(12, 2, 20, 5).sites)
    e, st = ctx.find_ground_state(ops, 20, s, 0.0, mixed(ctx))
    ref = golden["xxz_L12_D20_fields_seed5_E0"]
    assert abs(e - ref) <= TOL * abs(ref), (e, ref)
    assert st["split_rounds"] >= 1


def test_mixed_excited_state_and_gap(ctx, golden):
    ops = ctx.mpo(mo.ising_hmpo(10, 1, 1, 0))
    g = ctx.mps(mo.random_mps(10, 2, 16, 1).sites)
    x = ctx.mps(mo.random_mps(10, 2, 16, 11).sites)
    o = mixed(ctx)
    e0, s0 = ctx.find_ground_state(ops, 16, g, 0.0, o)
    e1, s1 = ctx.find_next_excited_state(ops, 16, [g], x, 0.0, o)
    r0, r1 = golden["ising_L10_D16_exc_E0"], golden["ising_L10_D16_exc_E1"]
    assert abs(e0 - r0) <= TOL * abs(r0)
    assert abs(e1 - r1) <= TOL * abs(r1), (e1, r1)
    assert abs((e1 - e0) - (r1 - r0)) <= TOL * abs(r1)
    assert s0["split_rounds"] >= 1 and s1["split_rounds"] >= 1
    assert abs(ctx.contract(x, None, g)) < 1e-6


def test_mixed_same_state_as_fp64(ctx):
    """Both paths end at the same state: local <sz> profiles agree to the
    observable bound."""
    H = mo.ising_hmpo(14, 1, 0.9, 0.05)
    m = ctx.mpo(H)
    a = ctx.mps(mo.random_mps(14, 2, 16, 8).sites)
    b = ctx.mps(mo.random_mps(14, 2, 16, 8).sites)
    ea, _ = ctx.find_ground_state(m, 16, a, 0.0, ctx.options(convtol=1e-10))
    eb, _ = ctx.find_ground_state(m, 16, b, 0.0, mixed(ctx))
    assert abs(ea - eb) <= TOL * abs(ea)
    sz = np.array([[1, 0], [0, -1]], dtype=complex)
    za = ctx.expectation_local(a, sz)
    zb = ctx.expectation_local(b, sz)
    np.testing.assert_allclose(zb, za, atol=1e-8)


def test_split_time_evolution_tracks_fp64(ctx):
    """optimize (the variational MPO.MPS step of time evolution) with
    precision 1 -- the local vector L W R x as a split-precision product,
    environments in FP64, each step converged to a relative distance change
    of 1e-6 (the products' noise floor) -- follows the FP64 evolution of a
    quench: after 10 real-time steps of an L=16 Ising chain at D<=16 the
    centre <sigma_x>, the centre-bond entropy and the energy agree with FP64
    to 1e-4.  This bound is the stated observable error of the split
    evolution, not the FP64 path's 1e-8."""
    L, D, g = 16, 16, 1.3
    U = ctx.mpo_ising_evolution(L, 1.0, g, 0.1, 0.02, False)
    H = ctx.mpo_ising(L, 1.0, g, 0.1)
    sx = np.array([[0, 1], [1, 0]], dtype=complex)
    out, split = {}, {}
    for prec in (0, 1):
        st = ctx.mps_product(L, 2, 1)
        o = ctx.options(convtol=1e-10, precision=prec)
        obs = []
        split[prec] = 0
        for _ in range(10):
            aux = st.copy()
            stats = ctx.optimize(U, aux, st, D, o)
            split[prec] += stats["split_matvecs"]
            aux.free()
            x = ctx.expectation_local(st, sx)[L // 2]
            st.gauge("L")
            obs.append((x, ctx.entropy(st, L // 2), ctx.contract(st, H, st).real))
        out[prec] = np.array(obs, dtype=float)
    np.testing.assert_allclose(out[1], out[0], rtol=0, atol=1e-4)
    assert split[0] == 0 and split[1] > 0
