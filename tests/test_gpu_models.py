"""GPU runs of the MPO builders beyond Ising and Schwinger: the Heisenberg
(XYZ) chain built by the library (bit-exact against the reference's tensors)
and its ground states against the reference's own runs (tests/golden)."""
import numpy as np
import pytest

from oracle import mps_oracle as mo

pytestmark = pytest.mark.gpu


def test_heisenberg_mpo_bit_exact(ctx, mpo_npz):
    ws = ctx.mpo_heisenberg(6, 1, 0.8, 1.2, 0.3, 0.1, 0.5, 0.7).download()
    for k in range(6):
        np.testing.assert_array_equal(ws[k], mpo_npz[f"heis6_{k}"])


@pytest.mark.parametrize("key,L,D,seed,params", [
    ("heisenberg_L10_D16_seed0_E0", 10, 16, 0, (1, 1, 1, 0, 0, 0)),
    ("xxz_L12_D20_fields_seed5_E0", 12, 20, 5, (1, 0.7, 1.3, 0.2, 0.1, 0.4)),
])
def test_heisenberg_gs_matches_reference(ctx, golden, key, L, D, seed, params):
    ops = ctx.mpo_heisenberg(L, *params)
    s = ctx.mps(mo.random_mps(L, 2, D, seed).sites)
    e, _ = ctx.find_ground_state(ops, D, s, 0.0, ctx.options(convtol=1e-10))
    ref = golden[key]
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)


def test_bosehubbard_mpo_and_ground_state(ctx, golden, mpo_npz):
    """Bose-Hubbard chain with up to two bosons per site (d = 3): the
    library's MPO equals the reference's tensors and the sweep from the
    seeded initial state reaches the reference's energy."""
    ws = ctx.mpo_bosehubbard(6, 2, 1.0, 2.0, 3, 0.25, 0.5).download()
    for k in range(6):
        np.testing.assert_array_equal(ws[k], mpo_npz[f"bh6_{k}"])
    ops = ctx.mpo_bosehubbard(8, 2, 1.0, 2.0, 4, 1.0, 0.0)
    s = ctx.mps(mo.random_mps(8, 3, 12, 6).sites)
    e, _ = ctx.find_ground_state(ops, 12, s, 0.0, ctx.options(convtol=1e-10))
    ref = golden["bosehubbard_L8_N2_D12_seed6_E0"]
    assert abs(e - ref) <= 1e-10 * abs(ref), (e, ref)
