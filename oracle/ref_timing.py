"""Timing the reference itself (oracle/_ref/ref_driver, the reference compiled
from its own sources) on this host's cores: the CPU baseline of bench.py and
its calibration.  Test infrastructure, like the rest of oracle/: bench.py's
cpu_baseline leg and --impl reference, and tests/golden/make_golden_large.py,
are its only callers.

The reference's complete solve of the headline workload (Schwinger N=100,
x=100, m/g=0.125, D=128, ground state from seed 1 and first excited state
from seed 11) was run once in full on one core of the build host: its wall
time and product counts are pinned in tests/golden/golden.json
(reference_timing).  A bounded sample measures how fast the reference runs on
another host: one bulk site step of the ground-state sweep per process
(environments set up untimed, then the site's eigensolve stopped after `cap`
products, its QR gauge move and its environment update, i.e. the reference's
own site step of Contractor::findGroundState, Contractor.cpp:1352-1533), at
positions spread over the chain's bulk, one single-threaded process per core.
The same sample, run on the build host when the full run was pinned, gives
the calibration rate; the full solve's time on this host is then the pinned
time scaled by the ratio of the two rates.
"""
import json
import os
import subprocess
import tempfile
import time

from oracle import mps_oracle as mo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.json")

N, D, X, MG, SEED = 100, 128, 100.0, 0.125, 1
MU = 2 * MG * X ** 0.5
CAP = 60                    # products of a sampled site step's eigensolve
FIRST, SPAN = 20, 60        # the sampled positions lie in sites FIRST .. FIRST + SPAN - 1


def pinned() -> dict:
    """The pinned full run (seconds and products of both phases) and the
    calibration rate, or None when not generated."""
    try:
        with open(GOLDEN) as f:
            t = json.load(f)["reference_timing"]
        return {"gs": t["schwinger_N100_D128_gs"], "exc": t["schwinger_N100_D128_exc"],
                "calibration": t.get("schwinger_N100_D128_calibration")}
    except (OSError, KeyError, ValueError):
        return None


def speed_sample(procs: int, cap: int = CAP) -> dict:
    """`procs` single-threaded reference processes at once, each timing one
    bulk site step with its eigensolve stopped after `cap` products; returns
    the products, core-seconds, products per core-second and wall time."""
    if not os.path.exists(DRIVER):
        raise FileNotFoundError("oracle/_ref/ref_driver not built (make -C oracle)")
    tmp = tempfile.mkdtemp()
    fn = os.path.join(tmp, "init.mps")
    mo.write_mps(fn, mo.random_mps(N, 2, D, SEED))
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1", ASAN_OPTIONS="detect_leaks=0", MPSDYN_SHIM_MAX_ITERS=str(cap))
    model = f"schwinger:{N}:{MU}:{X}:0:0"
    procs = max(1, procs)
    pos = [FIRST + (SPAN * p) // procs for p in range(procs)]
    t0 = time.time()
    ps = [subprocess.Popen([DRIVER, "profile", model, str(D), "0", fn, "1", str(p0)], stdout=subprocess.PIPE,
                           stderr=subprocess.DEVNULL, text=True, env=env) for p0 in pos]
    outs = [p.communicate()[0] for p in ps]
    wall = time.time() - t0
    res = [json.loads([l for l in o.splitlines() if l.startswith("{")][-1]) for o in outs]
    products = sum(r["iterations"] for r in res)
    core_s = sum(r["seconds"] for r in res)
    return {"products": products, "core_seconds": core_s, "rate": products / core_s, "wall": wall,
            "procs": len(res), "cap": cap, "positions": pos}


def solve_seconds_here(sample: dict, strict: bool = True) -> tuple:
    """One core's time for the complete solve on this host: the pinned full
    run's time scaled by calibration rate / this host's rate (same sample
    shape; strict=False also accepts another cap, for plumbing tests only).
    Returns (seconds, description) or (None, reason)."""
    p = pinned()
    if not p or not p.get("calibration"):
        return None, "the reference's pinned full run or its calibration is missing"
    cal = p["calibration"]
    if strict and cal["cap"] != sample["cap"]:
        return None, f"sample cap {sample['cap']} differs from the calibration's {cal['cap']}"
    full = p["gs"]["seconds"] + p["exc"]["seconds"]
    secs = full * cal["products_per_core_second"] / sample["rate"]
    why = (f"the reference's complete solve ({p['gs']['products']} + {p['exc']['products']} products) took "
           f"{full:.1f} s on one core of the build host, whose calibration sample ran "
           f"{cal['products_per_core_second']:.2f} products/core-s; this host ran {sample['rate']:.2f}")
    return secs, why
