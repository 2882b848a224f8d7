"""Regenerate the golden fixtures of tests/golden from the reference itself.

Runs oracle/_ref/ref_driver (the reference library compiled from its own
sources by oracle/Makefile, with the eigensolver shim of oracle/eigs_shim.cpp
above the dense branch) on seeded inputs and stores inputs and outputs as
small .npz/.json files.  Needs the reference tree (only in the build
container); the fixtures themselves travel with the repository.

    make -C oracle && python tests/golden/make_golden.py
    python tests/golden/make_golden.py --io-optsum   # only io_optsum.npz
"""
from __future__ import annotations

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


def run(*args) -> dict:
    # The bundled OpenBLAS 0.3.15 crashes intermittently in its threaded
    # kernels on these sizes; the reference runs single-threaded BLAS here.
    env = dict(os.environ, OPENBLAS_NUM_THREADS=os.environ.get("OPENBLAS_NUM_THREADS", "1"),
               ASAN_OPTIONS="detect_leaks=0")
    out = subprocess.run([DRIVER, *map(str, args)], capture_output=True, text=True, check=True, env=env)
    return json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])


def rand_c(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def io_and_optsum(tmp: str) -> None:
    """MPO files written by MPO::saveMPO (bytes, for byte-exact interop) and
    Contractor::optimizeSum results (state vectors, normfact) into
    io_optsum.npz; nothing else is touched."""
    out = {}
    for name, spec in [("ising6", "ising:6:1:1:0.3"), ("schwinger6", "schwinger:6:2.5:100:0:0")]:
        fn = os.path.join(tmp, name + ".mpo")
        run("savempo", spec, fn)
        with open(fn, "rb") as f:
            out[f"mpofile_{name}"] = np.frombuffer(f.read(), dtype=np.uint8)
    # unit-norm kets: with norms ~1e4 the reference's distance (a difference
    # of terms ~|M|^2) is rounding noise and its increase test exits 212
    k1, k2 = os.path.join(tmp, "k1.mps"), os.path.join(tmp, "k2.mps")
    for fn, seed in ((k1, 41), (k2, 42)):
        m = mo.random_mps(8, 2, 6, seed)
        m.sites[0] = m.sites[0] / np.linalg.norm(mo.mps_to_vector(m))
        mo.write_mps(fn, m)
    for tag, D, terms in [("sum2_D4", 4, [(k1, 0.7, 0.2), (k2, -0.3, 0.5)]), ("one_D3", 3, [(k1, 1.0, 0.0)])]:
        fi, fo = os.path.join(tmp, "oi.mps"), os.path.join(tmp, "oo.mps")
        mo.write_mps(fi, mo.random_mps(8, 2, D, 43))
        args = [a for t in terms for a in t]
        r = run("optsum", D, 1e-10, fi, fo, *args)
        res = mo.read_mps(fo)
        out[f"optsum_{tag}_vec"] = mo.mps_to_vector(res)
        out[f"optsum_{tag}_normfact"] = np.array(r["normfact"])
        out[f"optsum_{tag}_dims"] = np.array([a.shape for a in res.sites])
    np.savez_compressed(os.path.join(HERE, "io_optsum.npz"), **out)


def main() -> None:
    if len(sys.argv) > 1 and sys.argv[1] == "--io-optsum":
        io_and_optsum(tempfile.mkdtemp())
        return
    tmp = tempfile.mkdtemp()
    golden = {}

    # MPO builders (bit-exact targets)
    mpos = {}
    for name, spec in [("ising6", "ising:6:1:1:0.3"), ("schwinger6", "schwinger:6:2.5:100:0:0"),
                       ("heis6", "heis:6:1:0.8:1.2:0.3:0.1:0.5:0.7"),
                       ("bh6", "bh:6:2:1:2:3:0.25:0.5"), ("bh6x", "bh:6:3:0.7:1.3:4:0.3:0.15")]:
        run("mpo", spec, os.path.join(tmp, name + "_"))
        for k in range(6):
            mpos[f"{name}_{k}"] = mo.load_array(os.path.join(tmp, f"{name}_{k}.bin"))
    run("umpo", "ising:6:1:1:0.3", 0.01, 1, os.path.join(tmp, "uimag_"))
    run("umpo", "ising:6:1:1:0.3", 0.01, 0, os.path.join(tmp, "ureal_"))
    for k in range(6):
        mpos[f"uimag6_{k}"] = mo.load_array(os.path.join(tmp, f"uimag_{k}.bin"))
        mpos[f"ureal6_{k}"] = mo.load_array(os.path.join(tmp, f"ureal_{k}.bin"))
    np.savez_compressed(os.path.join(HERE, "mpo_tensors.npz"), **mpos)

    # Kernel-level products: matvec (plain and hermitian) and environments
    rng = np.random.default_rng(1234)
    ker = {}
    for tag, (d, w1, w2, Dl, Dr) in {"a": (2, 3, 3, 6, 7), "b": (2, 5, 5, 9, 4)}.items():
        L = rand_c(rng, (Dl, w1, Dl))
        W = rand_c(rng, (d, w1, d, w2))
        R = rand_c(rng, (Dr, w2, Dr))
        x = rand_c(rng, (d * Dl * Dr,))
        for n, a in [("L", L), ("W", W), ("R", R)]:
            mo.save_array(os.path.join(tmp, n + ".bin"), a)
        mo.save_array(os.path.join(tmp, "x.bin"), x.reshape(-1, 1))
        run("matvec", *(os.path.join(tmp, f) for f in ["L.bin", "W.bin", "R.bin", "x.bin", "y.bin"]), 0.75)
        y = mo.load_array(os.path.join(tmp, "y.bin")).reshape(-1, order="F")
        run("matvec_herm", *(os.path.join(tmp, f) for f in ["L.bin", "W.bin", "R.bin", "x.bin", "yh.bin"]))
        yh = mo.load_array(os.path.join(tmp, "yh.bin")).reshape(-1, order="F")
        ket = rand_c(rng, (d, Dl, Dr))
        bra = rand_c(rng, (d, Dl, Dr))
        mo.save_array(os.path.join(tmp, "ket.bin"), ket)
        mo.save_array(os.path.join(tmp, "bra.bin"), bra)
        TL = rand_c(rng, (Dl, w1, Dl))
        TR = rand_c(rng, (Dr, w2, Dr))
        mo.save_array(os.path.join(tmp, "TL.bin"), TL)
        mo.save_array(os.path.join(tmp, "TR.bin"), TR)
        run("envL", *(os.path.join(tmp, f) for f in ["TL.bin", "ket.bin", "W.bin", "bra.bin", "eL.bin"]))
        run("envR", *(os.path.join(tmp, f) for f in ["TR.bin", "ket.bin", "W.bin", "bra.bin", "eR.bin"]))
        ker.update({f"{tag}_L": L, f"{tag}_W": W, f"{tag}_R": R, f"{tag}_x": x, f"{tag}_y_off075": y,
                    f"{tag}_yherm": yh, f"{tag}_ket": ket, f"{tag}_bra": bra, f"{tag}_TL": TL,
                    f"{tag}_TR": TR, f"{tag}_envL": mo.load_array(os.path.join(tmp, "eL.bin")),
                    f"{tag}_envR": mo.load_array(os.path.join(tmp, "eR.bin"))})
    np.savez_compressed(os.path.join(HERE, "kernels.npz"), **ker)

    # Sweeps from seeded initial states (generator: oracle.mps_oracle.random_mps)
    def gs(spec, L, D, seed, convtol=1e-10, d=2):
        fn = os.path.join(tmp, f"init_{seed}.mps")
        mo.write_mps(fn, mo.random_mps(L, d, D, seed))
        return run("gs", spec, D, convtol, 0, fn, os.path.join(tmp, "out.mps"))["E0"]

    golden["ising_L10_D8_seed0_E0"] = gs("ising:10:1:1:0", 10, 8, 0)
    golden["ising_L20_D20_seed0_E0"] = gs("ising:20:1:1:0", 20, 20, 0)
    golden["ising_L12_D16_h01_seed3_E0"] = gs("ising:12:1:0.8:0.1", 12, 16, 3)
    mu = 2 * 0.125 * np.sqrt(100.0)
    golden["schwinger_N16_D24_seed1_E0"] = gs(f"schwinger:16:{mu}:100:0:0", 16, 24, 1)
    golden["heisenberg_L10_D16_seed0_E0"] = gs("heis:10:1:1:1:0:0:0:0", 10, 16, 0)
    golden["xxz_L12_D20_fields_seed5_E0"] = gs("heis:12:1:0.7:1.3:0.2:0.1:0.4:0", 12, 20, 5)
    golden["bosehubbard_L8_N2_D12_seed6_E0"] = gs("bh:8:2:1:2:4:1:0", 8, 12, 6, d=3)

    # Excited state (penalty L/2 = 5 is above the N=10 gap)
    f0 = os.path.join(tmp, "e0.mps")
    f1 = os.path.join(tmp, "e1.mps")
    mo.write_mps(f0, mo.random_mps(10, 2, 16, 1))
    mo.write_mps(f1, mo.random_mps(10, 2, 16, 11))
    r = run("exc", "ising:10:1:1:0", 16, 1e-10, 0, f0, f1, os.path.join(tmp, "o0"), os.path.join(tmp, "o1"))
    golden["ising_L10_D16_exc_E0"] = r["E0"]
    golden["ising_L10_D16_exc_E1"] = r["E1"]

    # Imaginary-time evolution from MPS(L, D, d) (testIsing.cpp:106-138)
    r = run("imag", "ising:10:1:1:0", 6, 20, 0.05, 1e-10)
    golden["ising_L10_D6_imag_dt005_energies"] = r["energies"]
    # the full imaginary-time phase of the L=20 Ising configuration
    # (testIsing.cpp with M = 200, delta = 0.01, D = 20)
    r = run("imag", "ising:20:1:1:0", 20, 200, 0.01, 1e-10)
    golden["ising_L20_D20_imag_dt001_M200_energies"] = r["energies"]

    # Real-time quench from |0...0> with D=1 initial bonds
    fq = os.path.join(tmp, "q.mps")
    mo.write_mps(fq, mo.product_mps(8, 2, 1))
    r = run("evolve", "ising:8:1:1.2:0.1", 8, 10, 0.05, 1e-10, fq, os.path.join(tmp, "qo.mps"))
    golden["ising_L8_D8_quench_sx_center"] = r["sx_center"]
    golden["ising_L8_D8_quench_energies"] = r["energies"]
    golden["ising_L8_D8_quench_entropy"] = r["entropy_center"]

    # SVD truncation MPS(mps, D) and MPO application (exact and cut), as
    # dense state vectors (gauge-invariant) with the site dimensions
    trunc = {}
    fi, fo = os.path.join(tmp, "t_in.mps"), os.path.join(tmp, "t_out.mps")
    mo.write_mps(fi, mo.random_mps(10, 2, 16, 21))
    run("truncate", fi, 5, fo)
    t = mo.read_mps(fo)
    trunc["trunc_L10_D16_seed21_to5_vec"] = mo.mps_to_vector(t)
    trunc["trunc_L10_D16_seed21_to5_dims"] = np.array([a.shape for a in t.sites])
    mo.write_mps(fi, mo.random_mps(8, 2, 6, 5))
    for D in (0, 4):
        for dg in (0, 1):
            for dr in "LR":
                run("applympo", "ising:8:1:1.1:0.2", 0.05, 0, D, dg, dr, fi, fo)
                t = mo.read_mps(fo)
                tag = f"apply_L8_D6_seed5_ureal005_cut{D}_dag{dg}_{dr}"
                trunc[tag + "_vec"] = mo.mps_to_vector(t)
                trunc[tag + "_dims"] = np.array([a.shape for a in t.sites])
    np.savez_compressed(os.path.join(HERE, "truncation.npz"), **trunc)
    # ground state from an initial MPS with a larger bond than D (the
    # prologue cuts it with MPS(init, D))
    fg = os.path.join(tmp, "g_in.mps")
    mo.write_mps(fg, mo.random_mps(12, 2, 16, 4))
    golden["ising_L12_init16_D6_seed4_E0"] = run("gs", "ising:12:1:1:0", 6, 1e-10, 0, fg,
                                                 os.path.join(tmp, "g_out.mps"))["E0"]

    # <psi|H^dag H|psi> (Contractor::contract2) and the errN / errT of one
    # optimize step
    fc = os.path.join(tmp, "c2.mps")
    mo.write_mps(fc, mo.random_mps(8, 2, 6, 7))
    golden["contract2_ising_L8_D6_seed7"] = run("contract2", "ising:8:1:1.1:0.2", fc)["re"]
    golden["contract2_schwinger_N8_D6_seed7"] = run("contract2", "schwinger:8:2.5:100:0:0", fc)["re"]
    mo.write_mps(fc, mo.random_state(8, 2, 6, 9))
    r = run("opterr", "ising:8:1:1.1:0.2", 0.05, 0, 6, fc)
    golden["opterr_ising_L8_D6_state9_ureal005"] = [r["errN"], r["errT"], r["normfact"]]

    io_and_optsum(tmp)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1)
    print(json.dumps({k: (v if not isinstance(v, list) else v[:3]) for k, v in golden.items()}, indent=1))


if __name__ == "__main__":
    main()
