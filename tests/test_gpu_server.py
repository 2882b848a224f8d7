"""GPU tests of the solve server (continuous batching): a request gives the
same result alone and in a mix of concurrently running requests, requests
are admitted by device footprint, and queued or running requests can be
cancelled."""
import time

import numpy as np
import pytest

from oracle import mps_oracle as mo

pytestmark = pytest.mark.gpu

ISING = 0


def _wait(srv, n, timeout=300):
    out = []
    t0 = time.time()
    while len(out) < n and time.time() - t0 < timeout:
        out.extend(srv.poll())
        time.sleep(0.01)
    return out


def test_same_result_alone_and_in_the_mix():
    from mpsdyn_b200 import capi
    probe = dict(model=ISING, L=12, D=16, p0=1.0, p1=0.9, p2=0.1, seed=77)
    with capi.Server(0, slots=1) as srv:
        srv.submit(**probe)
        alone = _wait(srv, 1)[0]
    with capi.Server(0, slots=4) as srv:
        ids = []
        for i, (L, D) in enumerate([(40, 32), (16, 8), (30, 24), (20, 16), (24, 32)]):
            ids.append(srv.submit(ISING, L, D, 1.0, 0.6 + 0.1 * i, 0.05, 100 + i))
            if i == 1:
                pid = srv.submit(**probe)
        res = {r["id"]: r for r in _wait(srv, 6)}
    assert alone["status"] == 0 and res[pid]["status"] == 0
    # same arithmetic on its own stream: identical to the last bit
    assert res[pid]["energy"] == alone["energy"]
    # and the ground state of that chain (oracle, same seeded initial state)
    e = mo.find_ground_state(mo.ising_hmpo(12, 1.0, 0.9, 0.1), 16, mo.random_mps(12, 2, 16, 77), convtol=1e-10)
    assert abs(alone["energy"] - e) <= 1e-10 * abs(e)
    assert all(r["status"] == 0 for r in res.values())
    # several requests were in flight at once
    spans = sorted((r["t_start"], r["t_end"]) for r in res.values())
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))


def test_admission_by_footprint():
    from mpsdyn_b200 import capi
    with capi.Server(0, slots=4, hbm_budget_bytes=1) as tmp:
        fp = tmp.footprint(ISING, 24, 32)
    # room for one request at a time although four slots are free
    with capi.Server(0, slots=4, hbm_budget_bytes=int(fp * 1.5)) as srv:
        for i in range(3):
            srv.submit(ISING, 24, 32, 1.0, 1.0, 0.0, 10 + i)
        res = sorted(_wait(srv, 3), key=lambda r: r["t_start"])
    assert all(r["status"] == 0 for r in res)
    for a, b in zip(res, res[1:]):
        assert b["t_start"] >= a["t_end"] - 1e-6
    with pytest.raises(capi.MpsgpuError):
        with capi.Server(0, slots=1, hbm_budget_bytes=fp // 2) as srv:
            srv.submit(ISING, 24, 32, 1.0, 1.0, 0.0, 1)


def test_cancel_queued_and_running():
    from mpsdyn_b200 import capi
    CANCELLED = 6
    with capi.Server(0, slots=1) as srv:
        long_id = srv.submit(1, 60, 64, 2.5, 100.0, 0.0, 3)   # Schwinger N=60, D=64: seconds
        queued_id = srv.submit(ISING, 10, 8, 1.0, 1.0, 0.0, 4)
        srv.cancel(queued_id)
        time.sleep(0.5)                                        # let the long one start
        srv.cancel(long_id)
        res = {r["id"]: r for r in _wait(srv, 2)}
    assert res[queued_id]["status"] == CANCELLED
    assert res[long_id]["status"] == CANCELLED
    assert res[long_id]["t_end"] - res[long_id]["t_start"] < 30


def test_first_fit_admission_passes_a_large_head():
    """A request too large for the memory left waits while smaller ones that
    fit start in the free slots (first fit, not head-of-line blocking)."""
    from mpsdyn_b200 import capi
    with capi.Server(0, slots=4, hbm_budget_bytes=1) as tmp:
        big = tmp.footprint(ISING, 60, 128)
        small = tmp.footprint(ISING, 16, 8)
    with capi.Server(0, slots=4, hbm_budget_bytes=1) as tmp:
        mid = tmp.footprint(ISING, 100, 64)
    assert mid > 2 * small and big + small >= mid
    budget = big + 2 * small  # room for the big one only when little else runs
    with capi.Server(0, slots=4, hbm_budget_bytes=budget) as srv:
        first = srv.submit(ISING, 100, 64, 1.0, 1.0, 0.0, 5)   # occupies memory for a while
        big_id = srv.submit(ISING, 60, 128, 1.0, 1.0, 0.0, 6)  # cannot start next to it
        small_ids = [srv.submit(ISING, 16, 8, 1.0, 0.9, 0.0, 20 + i) for i in range(2)]
        res = {r["id"]: r for r in _wait(srv, 4, timeout=600)}
    assert all(r["status"] == 0 for r in res.values())
    # the small requests started before the large one that was queued ahead of them
    assert all(res[i]["t_start"] < res[big_id]["t_start"] for i in small_ids)
    assert res[first]["status"] == 0


def test_time_evolution_request_alone_and_in_the_mix(tmp_path):
    """A served quench gives the same observables alone and next to other
    requests, equal to the library called directly, and writes its final
    state to the requested file."""
    from mpsdyn_b200 import capi
    L, D, g, steps = 16, 16, 1.3, 6
    with capi.Server(0, slots=1) as srv:
        rid, sx_a, ent_a = srv.submit_evolution(L, D, 1.0, g, 0.1, steps, 0.05)
        alone = _wait(srv, 1)[0]
    out = tmp_path / "final.mps"
    with capi.Server(0, slots=3) as srv:
        ids = [srv.submit(ISING, 30, 24, 1.0, 0.8, 0.1, 50)]
        rid2, sx_b, ent_b = srv.submit_evolution(L, D, 1.0, g, 0.1, steps, 0.05, result_file=out)
        ids.append(srv.submit(ISING, 24, 16, 1.0, 1.1, 0.0, 51))
        res = {r["id"]: r for r in _wait(srv, 3)}
    assert alone["status"] == 0 and res[rid2]["status"] == 0
    np.testing.assert_array_equal(sx_a, sx_b)
    np.testing.assert_array_equal(ent_a, ent_b)
    assert res[rid2]["energy"] == alone["energy"]
    # against the library's own calls (the quench loop of the batched workload)
    with capi.Context(0) as c:
        U = c.mpo_ising_evolution(L, 1.0, g, 0.1, 0.05, False)
        st = c.mps_product(L, 2, 1)
        o = c.options(convtol=1e-10)
        for k in range(steps):
            aux = st.copy()
            c.optimize(U, aux, st, D, o)
            aux.free()
            assert c.expectation_local(st, mo.SIGX)[L // 2] == sx_a[k]
            st.gauge("L")
            assert c.entropy(st, L // 2) == ent_a[k]
        saved = c.mps_import(out)
        H = c.mpo_ising(L, 1.0, g, 0.1)
        e = c.contract(saved, H, saved).real / c.contract(saved, None, saved).real
        assert abs(e - alone["energy"]) <= 1e-10 * abs(e)
