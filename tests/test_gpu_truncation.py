"""GPU parity of the SVD-cut paths: MPS(mps, D) (MPS.cpp:761-772), MPO
application exact or cut (MPS::applyExactly / MPS::truncate, MPS.cpp:
858-936), and the findGroundState prologue that cuts an initial state with
a larger bond.  States are compared as dense vectors (the SVD leaves a
phase per kept singular vector free), site dimensions bit-exact, against
fixtures written by the reference itself (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from oracle import mps_oracle as mo

pytestmark = pytest.mark.gpu


def dev_state(s):
    sites, nf = s.download()
    return mo.MPS([np.asarray(a) for a in sites], nf)


def test_approximate_matches_reference(ctx, trunc_npz):
    m = mo.random_mps(10, 2, 16, 21)
    s = ctx.mps(m.sites)
    t, disc = s.approximate(5)
    r = dev_state(t)
    np.testing.assert_array_equal(np.array([a.shape for a in r.sites]), trunc_npz["trunc_L10_D16_seed21_to5_dims"])
    ref = trunc_npz["trunc_L10_D16_seed21_to5_vec"]
    assert np.abs(mo.mps_to_vector(r) - ref).max() < 1e-12 * np.abs(ref).max()
    # discarded weight (not reported by the reference) against the oracle
    o = mo.truncate_mps(m, 5)
    assert abs(disc - sum(o.discarded)) < 1e-10 * max(1.0, sum(o.discarded))


@pytest.mark.parametrize("cut", [0, 4])
@pytest.mark.parametrize("dagger", [0, 1])
@pytest.mark.parametrize("direction", ["L", "R"])
def test_apply_mpo_matches_reference(ctx, trunc_npz, cut, dagger, direction):
    U = ctx.mpo(mo.ising_umpo(8, 1.0, 1.1, 0.2, 0.05, False))
    s = ctx.mps(mo.random_mps(8, 2, 6, 5).sites)
    t, disc = s.apply_mpo(U, cut, bool(dagger), direction)
    r = dev_state(t)
    tag = f"apply_L8_D6_seed5_ureal005_cut{cut}_dag{dagger}_{direction}"
    np.testing.assert_array_equal(np.array([a.shape for a in r.sites]), trunc_npz[tag + "_dims"])
    ref = trunc_npz[tag + "_vec"]
    assert np.abs(mo.mps_to_vector(r) - ref).max() < 1e-12 * np.abs(ref).max()
    if cut == 0:
        assert disc < 1e-20


def test_apply_mpo_larger_bonds_vs_oracle(ctx):
    # D = 40 state, w = 4 operator: SVDs of up to 160 x 80 on the device
    L = 10
    m = mo.random_state(L, 2, 40, 8)
    Uh = mo.ising_umpo(L, 1.0, 0.9, 0.1, 0.02, False)
    s = ctx.mps(m.sites, m.normfact)
    U = ctx.mpo(Uh)
    for cut in (0, 24):
        t, disc = s.apply_mpo(U, cut, False, "L")
        r = dev_state(t)
        o = mo.apply_mpo(Uh, m, cut, False, "L")
        assert [a.shape for a in r.sites] == [a.shape for a in o.sites]
        vo = mo.mps_to_vector(o)
        assert np.abs(mo.mps_to_vector(r) - vo).max() < 1e-11 * np.abs(vo).max()
        assert abs(disc - o.discarded) < 1e-10 * max(1.0, o.discarded)


def test_gs_prologue_truncates_large_initial_bond(ctx, golden):
    ops = ctx.mpo(mo.ising_hmpo(12, 1, 1, 0))
    s = ctx.mps(mo.random_mps(12, 2, 16, 4).sites)
    e, _ = ctx.find_ground_state(ops, 6, s, 0.0, ctx.options(convtol=1e-10))
    ref = golden["ising_L12_init16_D6_seed4_E0"]
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)


def test_svd_zero_values_dropped(ctx):
    # a zero-padded product state: every cut keeps only the nonzero value
    m = mo.product_mps(8, 2, 1)
    mo.increase_bond_dimension(m, 4)
    s = ctx.mps(m.sites)
    t, disc = s.approximate(3)
    r = dev_state(t)
    assert all(a.shape[1] == 1 and a.shape[2] == 1 for a in r.sites)
    assert disc == 0.0
    assert abs(abs(mo.mps_to_vector(r)[0]) - 1.0) < 1e-14
