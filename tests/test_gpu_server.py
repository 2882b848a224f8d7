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
