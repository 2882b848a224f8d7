"""A bounded sample of the headline sweep for profilers.

    python -m mpsdyn_b200.profile_sample [--sites 40] [--D 128] [--rounds 1]

Runs the ground-state sweep of the Schwinger chain (x = 100, m/g = 0.125,
mu = 2.5, seed-1 initial MPS, convergence 1e-10) on `--sites` sites with bond
`--D`, stopped after `--rounds` half-sweeps (the library returns
MPSGPU_NOT_CONVERGED at the round limit, which ends the sample).  With 40
sites, 26 bulk sites have the (128, 5, 128) shapes of the 100-site chain, so
the kernel mix per site step is the headline's while the launch count stays
small enough for a profiler that slows every launch down.  Prints one JSON
line (launches, site solves, products, seconds).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from mpsdyn_b200 import capi


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--sites", type=int, default=40)
    p.add_argument("--D", type=int, default=128)
    p.add_argument("--rounds", type=int, default=1)
    a = p.parse_args()
    mu = 2 * 0.125 * np.sqrt(100.0)
    with capi.Context(0) as ctx:
        H = ctx.mpo_schwinger(a.sites, mu, 100.0)
        psi = ctx.mps_random(a.sites, 2, a.D, 1)
        o = ctx.options(convtol=1e-10, max_rounds=a.rounds)
        l0 = ctx.launches
        t0 = time.perf_counter()
        status = "converged"
        try:
            ctx.find_ground_state(H, a.D, psi, 0.0, o)
        except capi.MpsgpuError as e:
            if e.status != 2:  # anything but the round limit is a failure
                raise
            status = "round limit"
        ctx.synchronize()
        print(json.dumps({"sample": f"schwinger N={a.sites} D={a.D}, {a.rounds} half-sweep(s)", "status": status,
                          "launches": ctx.launches - l0, "seconds": time.perf_counter() - t0}), flush=True)


if __name__ == "__main__":
    main()
