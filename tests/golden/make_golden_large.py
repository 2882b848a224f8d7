"""Pinned reference results at the sizes that are timed (long CPU jobs).

Runs oracle/_ref/ref_driver (the reference library compiled from its own
sources by oracle/Makefile, eigensolver shim above the dense branch) on the
seeded inputs of three workloads and merges the results into
tests/golden/golden.json (keys below); the other fixtures are untouched.

  schwinger_N100_D128_seed1_E0 / _seed11_E1 / _gap
      SchwingerHamiltonian(100, mu=2.5, x=100, 0, 0), D = 128, convtol 1e-10:
      findGroundState from the seed-1 MPS, findNextExcitedState from the
      seed-11 MPS (Contractor.cpp:1352-1533, 2676-2727); also the reference's
      wall time and product counts of both phases ("reference_timing").
      About 1.5 h per phase on one core.
  ising_L128_D64_g1_h01_seed7_E0
      IsingHamiltonian(128, 2, J=1, g=1, h=0.1), D = 64, convtol 1e-10,
      seed-7 MPS (a request of the serving mix).  About 10 min.
  quench_L64_D64_g1649_h01_dt001_{sx_center,entropy_center,energies}
      real-time evolution of the open Ising chain L = 64, J = 1,
      g = 1.6490052627416842 (the first draw of numpy's default_rng(5) on
      U[0.2, 2.0], as the batched quench workload draws it), h = 0.1, from
      |0...0> at D = 1, second-order U-MPO with dt = 0.01, 20 steps at
      D <= 64 (flatIsing.cpp:174-205 as ref_driver's `evolve`).

    make -C oracle && python tests/golden/make_golden_large.py [--jobs 3]
    python tests/golden/make_golden_large.py --from-logs DIR   # parse logs of an earlier run

The three jobs run as parallel single-threaded processes; their stdout goes
to DIR/<name>.log (a temporary directory unless --logs is given).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import mps_oracle as mo  # noqa: E402

DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
MU = 2 * 0.125 * np.sqrt(100.0)
G_QUENCH = float(np.random.default_rng(5).uniform(0.2, 2.0, size=64)[0])

JOBS = {
    "schwinger_exc": lambda d: ["exc", f"schwinger:100:{MU}:100:0:0", 128, 1e-10, 0,
                                os.path.join(d, "schw_seed1.mps"), os.path.join(d, "schw_seed11.mps"),
                                os.path.join(d, "schw_gs.mps"), os.path.join(d, "schw_exc.mps")],
    "ising_L128": lambda d: ["gs", "ising:128:1:1.0:0.1", 64, 1e-10, 0, os.path.join(d, "ising128_seed7.mps"),
                             os.path.join(d, "ising128_out.mps")],
    "quench_L64": lambda d: ["evolve", f"ising:64:1:{G_QUENCH!r}:0.1", 64, 20, 0.01, 1e-10,
                             os.path.join(d, "quench_init.mps"), os.path.join(d, "quench_out.mps")],
}


def write_inputs(d: str) -> None:
    mo.write_mps(os.path.join(d, "schw_seed1.mps"), mo.random_mps(100, 2, 128, 1))
    mo.write_mps(os.path.join(d, "schw_seed11.mps"), mo.random_mps(100, 2, 128, 11))
    mo.write_mps(os.path.join(d, "ising128_seed7.mps"), mo.random_mps(128, 2, 64, 7))
    mo.write_mps(os.path.join(d, "quench_init.mps"), mo.product_mps(64, 2, 1))


def last_json(path: str) -> dict:
    with open(path) as f:
        return json.loads([l for l in f.read().splitlines() if l.startswith("{")][-1])


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--from-logs", default=None, help="parse <name>.log files of an earlier run")
    ap.add_argument("--logs", default=None, help="directory for the logs and inputs (default: a temp dir)")
    ap.add_argument("--calibrate", action="store_true",
                    help="only time the bounded speed sample of oracle/ref_timing.py on this host (all cores) and "
                         "store it next to the full run it calibrates")
    a = ap.parse_args()
    if a.calibrate:
        from oracle import ref_timing
        s = ref_timing.speed_sample(os.cpu_count() or 1)
        gfile = os.path.join(HERE, "golden.json")
        with open(gfile) as f:
            golden = json.load(f)
        golden.setdefault("reference_timing", {})["schwinger_N100_D128_calibration"] = {
            "products_per_core_second": s["rate"], "cap": s["cap"], "procs": s["procs"],
            "products": s["products"], "core_seconds": s["core_seconds"], "positions": s["positions"],
            "note": "oracle/ref_timing.speed_sample on the host of the full run, all its cores"}
        with open(gfile, "w") as f:
            json.dump(golden, f, indent=1)
        print(json.dumps(golden["reference_timing"]["schwinger_N100_D128_calibration"]))
        return
    if a.from_logs:
        d = a.from_logs
    else:
        d = a.logs or tempfile.mkdtemp()
        os.makedirs(d, exist_ok=True)
        write_inputs(d)
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1", ASAN_OPTIONS="detect_leaks=0")
        procs = {name: subprocess.Popen([DRIVER, *map(str, make(d))], stdout=open(os.path.join(d, name + ".log"), "w"),
                                        stderr=subprocess.STDOUT, env=env)
                 for name, make in JOBS.items()}
        for name, p in procs.items():
            if p.wait() != 0:
                raise SystemExit(f"{name}: ref_driver exited {p.returncode}")
    def result(name):
        # a job whose log has no final JSON line (still running) is skipped
        try:
            return last_json(os.path.join(d, name + ".log"))
        except (OSError, IndexError, ValueError):
            print(f"{name}: no result yet, left out")
            return None
    r_exc, r_is, r_q = result("schwinger_exc"), result("ising_L128"), result("quench_L64")
    gfile = os.path.join(HERE, "golden.json")
    with open(gfile) as f:
        golden = json.load(f)
    timing = golden.get("reference_timing", {
        "note": "reference compiled from source (oracle/_ref), one core, single-threaded OpenBLAS, "
                "eigensolver shim; seconds and effective-Hamiltonian products per phase"})
    if r_exc:
        golden["schwinger_N100_D128_seed1_E0"] = r_exc["E0"]
        golden["schwinger_N100_D128_seed11_E1"] = r_exc["E1"]
        golden["schwinger_N100_D128_gap"] = r_exc["gap"]
        timing["schwinger_N100_D128_gs"] = {"seconds": r_exc["gs_seconds"], "products": r_exc["gs_products"],
                                            "site_solves": r_exc["gs_site_solves"]}
        timing["schwinger_N100_D128_exc"] = {"seconds": r_exc["exc_seconds"], "products": r_exc["exc_products"],
                                             "site_solves": r_exc["exc_site_solves"]}
    if r_is:
        golden["ising_L128_D64_g1_h01_seed7_E0"] = r_is["E0"]
        timing["ising_L128_D64_gs"] = {"seconds": r_is["seconds"], "products": r_is["products"],
                                       "site_solves": r_is["site_solves"]}
    if r_q:
        golden["quench_L64_D64_g1649_h01_dt001_sx_center"] = r_q["sx_center"]
        golden["quench_L64_D64_g1649_h01_dt001_entropy_center"] = r_q["entropy_center"]
        golden["quench_L64_D64_g1649_h01_dt001_energies"] = r_q["energies"]
    golden["reference_timing"] = timing
    with open(gfile, "w") as f:
        json.dump(golden, f, indent=1)
    print(json.dumps({k: golden.get(k) for k in ("schwinger_N100_D128_seed1_E0", "schwinger_N100_D128_seed11_E1",
                                                "ising_L128_D64_g1_h01_seed7_E0", "reference_timing")}, indent=1))


if __name__ == "__main__":
    main()
