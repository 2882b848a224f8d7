"""GPU tests of the file formats, checkpoints and optimizeSum.

* MPO::saveMPO / loadMPO (MPO.cpp:214-231, 291-312): the library writes
  byte-identical files to the reference's (fixtures written by the reference
  itself, tests/golden/io_optsum.npz) and loads them back bit-exactly;
* MPS::exportMPS / importMPS (MPS.cpp:442-509): byte-identical to the
  oracle's writer of the same format, and a round trip;
* checkpoints of findGroundState (tmpfile / freqSv, Contractor.cpp:1526-1530):
  a solve cut off after two half-sweeps leaves a state file from which a
  second call reaches the same energy as an uninterrupted solve and the
  reference (|dE/E| <= 1e-10);
* the excited-state sweep saves at the end of every half-sweep
  (Contractor.cpp:2868-2883);
* Contractor::optimizeSum / optimizeMPS (Contractor.cpp:2319-2477) against
  the reference's results (state vectors 1e-10, dimensions bit-exact).
"""
import os

import numpy as np
import pytest

from oracle import mps_oracle as mo

pytestmark = pytest.mark.gpu

MU = 2 * 0.125 * np.sqrt(100.0)


@pytest.fixture(scope="module")
def io_npz():
    here = os.path.join(os.path.dirname(__file__), "golden", "io_optsum.npz")
    return np.load(here)


def _parse_mpo_file(b: bytes):
    L = int(np.frombuffer(b[:4], dtype=np.int32)[0])
    off, out = 4, []
    for _ in range(L):
        rank = int(np.frombuffer(b[off:off + 4], dtype=np.int32)[0])
        dims = tuple(np.frombuffer(b[off + 4:off + 4 + 4 * rank], dtype=np.int32))
        off += 4 + 4 * rank
        n = int(np.prod(dims))
        out.append((dims, np.frombuffer(b[off:off + 16 * n], dtype=np.complex128)))
        off += 16 * n
    assert off == len(b)
    return out


def test_mpo_file_matches_reference(ctx, io_npz, tmp_path):
    # Ising: the same bytes as MPO::saveMPO writes
    fn = tmp_path / "ising6.mpo"
    ctx.mpo_save(ctx.mpo(mo.ising_hmpo(6, 1, 1, 0.3)), fn)
    assert fn.read_bytes() == io_npz["mpofile_ising6"].tobytes()
    # Schwinger: the same layout and values; the reference's BLAS product
    # C . Z (SchwingerHamiltonian.cpp:113-116) leaves -0.0 in two entries of
    # the first operator where the library's builder writes +0.0
    fn = tmp_path / "schwinger6.mpo"
    ctx.mpo_save(ctx.mpo_schwinger(6, MU, 100.0), fn)
    got, ref = _parse_mpo_file(fn.read_bytes()), _parse_mpo_file(io_npz["mpofile_schwinger6"].tobytes())
    assert len(got) == len(ref)
    for (dg, vg), (dr, vr) in zip(got, ref):
        assert dg == dr
        assert np.array_equal(vg, vr)


def test_mpo_load_reference_file(ctx, io_npz, tmp_path, mpo_npz):
    fn = tmp_path / "ref_ising6.mpo"
    fn.write_bytes(io_npz["mpofile_ising6"].tobytes())
    m = ctx.mpo_load(fn)
    for k, W in enumerate(m.download()):
        np.testing.assert_array_equal(W, mpo_npz[f"ising6_{k}"])


def test_mps_export_import(ctx, tmp_path):
    ref = mo.random_mps(7, 2, 5, 12)
    s = ctx.mps(ref.sites, 0.75)
    fn = tmp_path / "s.mps"
    ctx.mps_export(s, fn)
    ofn = tmp_path / "o.mps"
    ref.normfact = 0.75
    mo.write_mps(str(ofn), ref)
    b_lib, b_ora = fn.read_bytes(), ofn.read_bytes()
    # header bond/gauge fields come from the state's bookkeeping; the sites
    # (everything after the 20-byte header) are the same bytes
    assert b_lib[20:] == b_ora[20:]
    t = ctx.mps_import(fn)
    sites, nf = t.download()
    assert nf == 0.75
    for a, b in zip(sites, ref.sites):
        np.testing.assert_array_equal(a, b)


def test_ground_state_checkpoint_and_resume(ctx, golden, tmp_path):
    ops = mo.ising_hmpo(20, 1, 1, 0)
    init = mo.random_mps(20, 2, 20, 0)
    ref = golden["ising_L20_D20_seed0_E0"]
    ck = tmp_path / "gs.ckpt"
    m = ctx.mpo(ops)
    s = ctx.mps(init.sites)
    with pytest.raises(Exception):  # stopped by the round limit after two half-sweeps
        ctx.find_ground_state(m, 20, s, 0.0, ctx.options(convtol=1e-10, max_rounds=2, checkpoint_file=ck,
                                                           checkpoint_every=1))
    assert ck.exists() and ck.stat().st_size > 0
    resumed = ctx.mps_import(ck)
    e1, _ = ctx.find_ground_state(m, 20, resumed, 0.0, ctx.options(convtol=1e-10))
    full = ctx.mps(init.sites)
    e0, _ = ctx.find_ground_state(m, 20, full, 0.0, ctx.options(convtol=1e-10))
    assert abs(e1 - e0) <= 1e-10 * abs(e0), (e1, e0)
    assert abs(e1 - ref) <= 1e-10 * abs(ref), (e1, ref)


def test_excited_state_checkpoint_every_half_sweep(ctx, golden, tmp_path):
    ops = ctx.mpo(mo.ising_hmpo(10, 1, 1, 0))
    g = ctx.mps(mo.random_mps(10, 2, 16, 1).sites)
    ctx.find_ground_state(ops, 16, g, 0.0, ctx.options(convtol=1e-10))
    x = ctx.mps(mo.random_mps(10, 2, 16, 11).sites)
    ck = tmp_path / "exc.ckpt"
    e1, _ = ctx.find_next_excited_state(ops, 16, [g], x, 0.0, ctx.options(convtol=1e-10, checkpoint_file=ck))
    assert abs(e1 - golden["ising_L10_D16_exc_E1"]) <= 1e-10 * abs(e1)
    saved = ctx.mps_import(ck)  # the state at the end of the last half-sweep
    es = ctx.contract(saved, ops, saved).real / ctx.contract(saved, None, saved).real
    assert abs(es - e1) <= 1e-8 * abs(e1)


def _unit(seed):
    m = mo.random_mps(8, 2, 6, seed)
    m.sites[0] = m.sites[0] / np.linalg.norm(mo.mps_to_vector(m))
    return m


@pytest.mark.parametrize("tag,D,terms", [("sum2_D4", 4, [(41, 0.7 + 0.2j), (42, -0.3 + 0.5j)]),
                                          ("one_D3", 3, [(41, 1.0 + 0.0j)])])
def test_optimize_sum_matches_reference(ctx, io_npz, tag, D, terms):
    kets = [ctx.mps(_unit(seed).sites) for seed, _ in terms]
    init = ctx.mps(mo.random_mps(8, 2, D, 43).sites)
    ctx.optimize_sum(kets, [b for _, b in terms], init, D, ctx.options(convtol=1e-10))
    sites, nf = init.download()
    r = mo.MPS([np.asarray(a) for a in sites], nf)
    np.testing.assert_array_equal(np.array([a.shape for a in r.sites]), io_npz[f"optsum_{tag}_dims"])
    ref = io_npz[f"optsum_{tag}_vec"]
    assert np.abs(mo.mps_to_vector(r) - ref).max() < 1e-10 * np.abs(ref).max()
    assert abs(nf - float(io_npz[f"optsum_{tag}_normfact"])) < 1e-10


def test_optimize_mps_error(ctx):
    ket = ctx.mps(_unit(41).sites)
    init = ctx.mps(mo.random_mps(8, 2, 8, 44).sites)
    err, st = ctx.optimize_mps(ket, init, 8, ctx.options(convtol=1e-12))
    # D = 8 holds the D = 6 ket exactly
    assert abs(err) < 1e-10 and st["rounds"] >= 1
