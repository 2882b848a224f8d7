"""GPU tests of batched solves (mpsgpu_find_ground_state_batch /
mpsgpu_find_next_excited_state_batch): chains of different models and sizes
swept in lockstep on one stream, their local eigenproblems solved in shared
grouped launches, each reaching the energy the reference reaches for it
(tests/golden/golden.json, |dE/E| <= 1e-10) and the energy of the same solve
run alone (1e-10: the grouped last contraction may split its K range
differently than a single solve does, which changes rounding only, and the
sweeps then end within the convergence tolerance of each other)."""
import numpy as np
import pytest

from oracle import mps_oracle as mo

pytestmark = pytest.mark.gpu

MU = 2 * 0.125 * np.sqrt(100.0)

CASES = [  # (golden key, MPO tensors, initial MPS, D)
    ("ising_L10_D8_seed0_E0", lambda: mo.ising_hmpo(10, 1, 1, 0), lambda: mo.random_mps(10, 2, 8, 0), 8),
    ("ising_L12_D16_h01_seed3_E0", lambda: mo.ising_hmpo(12, 1, 0.8, 0.1), lambda: mo.random_mps(12, 2, 16, 3), 16),
    ("schwinger_N16_D24_seed1_E0", lambda: mo.schwinger_hmpo(16, MU, 100.0), lambda: mo.random_mps(16, 2, 24, 1), 24),
]


@pytest.mark.parametrize("precision", [0, 1])
def test_ground_state_batch_matches_reference_and_single(ctx, golden, precision):
    o = ctx.options(convtol=1e-10, precision=precision)
    ops = [ctx.mpo(mk()) for _, mk, _, _ in CASES]
    # the batch takes one bond dimension: every case at its own D through
    # separate batches of one, and all together at the common D = 24 below
    singles = []
    for (key, _, mps, D), m in zip(CASES, ops):
        s = ctx.mps(mps().sites)
        e, st = ctx.find_ground_state(m, D, s, 0.0, o)
        assert abs(e - golden[key]) <= 1e-10 * abs(golden[key]), (key, e)
        singles.append(e)
    for (key, _, mps, D), m, e1 in zip(CASES, ops, singles):
        inits = [ctx.mps(mps().sites) for _ in range(3)]
        es, stv, sts = ctx.find_ground_state_batch([m] * 3, D, inits, 0.0, o)
        assert stv == [0, 0, 0]
        for e in es:
            assert abs(e - golden[key]) <= 1e-10 * abs(golden[key]), (key, e)
            assert abs(e - e1) <= 1e-10 * abs(e1), (key, e, e1)
        assert all(x["matvecs"] > 0 for x in sts)


def test_ground_state_batch_of_different_chains(ctx, golden):
    # chains of different lengths and models in one batch at a common D
    o = ctx.options(convtol=1e-10)
    D = 8
    cases = [(mo.ising_hmpo(10, 1, 1, 0), mo.random_mps(10, 2, D, 0)),
             (mo.ising_hmpo(12, 1, 0.7, 0), mo.random_mps(12, 2, D, 9)),
             (mo.schwinger_hmpo(16, MU, 100.0), mo.random_mps(16, 2, D, 1))]
    ops = [ctx.mpo(m) for m, _ in cases]
    inits = [ctx.mps(s.sites) for _, s in cases]
    es, stv, _ = ctx.find_ground_state_batch(ops, D, inits, 0.0, o)
    assert stv == [0, 0, 0]
    assert abs(es[0] - golden["ising_L10_D8_seed0_E0"]) <= 1e-10 * abs(es[0])
    for (m, s), e in zip(cases[1:], es[1:]):
        alone = ctx.mps(s.sites)
        e1, _ = ctx.find_ground_state(ctx.mpo(m), D, alone, 0.0, o)
        assert abs(e - e1) <= 1e-10 * abs(e1)
    # the returned states are the ground states: <H> matches
    for m, s, e in zip(ops, inits, es):
        assert abs(ctx.contract(s, m, s).real - e) < 1e-9 * abs(e)


def test_excited_state_batch_matches_reference(ctx, golden):
    o = ctx.options(convtol=1e-10)
    m = ctx.mpo(mo.ising_hmpo(10, 1, 1, 0))
    gs = [ctx.mps(mo.random_mps(10, 2, 16, 1).sites) for _ in range(2)]
    es0, st0, _ = ctx.find_ground_state_batch([m, m], 16, gs, 0.0, o)
    assert st0 == [0, 0]
    xs = [ctx.mps(mo.random_mps(10, 2, 16, 11).sites) for _ in range(2)]
    es1, st1, sts = ctx.find_next_excited_state_batch([m, m], 16, [[gs[0]], [gs[1]]], xs, 0.0, o)
    assert st1 == [0, 0]
    r0, r1 = golden["ising_L10_D16_exc_E0"], golden["ising_L10_D16_exc_E1"]
    for e0, e1 in zip(es0, es1):
        assert abs(e0 - r0) <= 1e-10 * abs(r0)
        assert abs(e1 - r1) <= 1e-10 * abs(r1), (e1, r1)
    for x, g in zip(xs, gs):
        assert abs(ctx.contract(x, None, g)) < 1e-6
