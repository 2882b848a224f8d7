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
