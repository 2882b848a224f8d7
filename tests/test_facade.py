"""The C++ facade (mpsdyn_b200/cpp): reference class names and call
signatures over the C ABI.

CPU: the facade library builds, a program written against the reference's
API compiles and links against it, and - where the reference tree is
present - the reference's own programs/ising/testIsing.cpp compiles and links
against it unchanged (a source-level drop-in check).

GPU: that program runs the reference's call sequence (findGroundState,
testIsing's imaginary-time loop, findNextExcitedState, MPS(mps, D),
exportMPS/importMPS, contract2, getEntropy) and reproduces the reference's
own numbers from tests/golden.
"""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import mps_oracle as mo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "mpsdyn_b200")
INC = [os.path.join(PKG, "cpp", "include"), os.path.join(ROOT, "include")]
REF_TEST_ISING = "/root/reference/src/programs/ising/testIsing.cpp"


def _facade_lib():
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    lib = os.path.join(PKG, "libmpsdyn_facade.so")
    if not os.path.exists(lib):
        if shutil.which("nvcc") is None:
            pytest.skip("library not built and nvcc not available")
        from mpsdyn_b200 import build
        build.build()
    return lib


def _compile(src, out):
    cmd = ["g++", "-std=c++17", "-O1", *("-I" + i for i in INC), src, "-o", out, "-L" + PKG,
           "-lmpsdyn_facade", "-lmpsgpu", "-Wl,-rpath," + PKG]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return out


def test_program_compiles_against_facade(tmp_path):
    _facade_lib()
    _compile(os.path.join(ROOT, "tests", "native", "facade_program.cpp"), str(tmp_path / "facade_program"))


@pytest.mark.skipif(not os.path.exists(REF_TEST_ISING), reason="reference tree not present")
def test_reference_testIsing_compiles_unchanged(tmp_path):
    _facade_lib()
    _compile(REF_TEST_ISING, str(tmp_path / "testIsing"))


@pytest.mark.gpu
def test_facade_program_reproduces_reference(tmp_path, golden):
    _facade_lib()
    exe = _compile(os.path.join(ROOT, "tests", "native", "facade_program.cpp"), str(tmp_path / "facade_program"))
    files = []
    for name, m in (("gs", mo.random_mps(10, 2, 8, 0)), ("e0", mo.random_mps(10, 2, 16, 1)),
                    ("e1", mo.random_mps(10, 2, 16, 11)), ("tr", mo.random_mps(10, 2, 16, 21))):
        fn = str(tmp_path / f"{name}.mps")
        mo.write_mps(fn, m)
        files.append(fn)
    r = subprocess.run([exe, *files, str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    res = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    ref = golden["ising_L10_D8_seed0_E0"]
    assert abs(res["gs_E0"] - ref) <= 1e-10 * abs(ref)
    assert abs(res["mixed_gs_E0"] - ref) <= 1e-10 * abs(ref)
    assert abs(res["gs_norm"] - 1.0) < 1e-12
    assert abs(res["gs_H"] - res["gs_E0"]) < 1e-9 * abs(ref)
    # the ground state is an eigenstate: <H^2> = E^2
    assert abs(res["gs_H2"] - res["gs_E0"] ** 2) < 1e-8 * ref ** 2
    assert abs(res["roundtrip_overlap"] - 1.0) < 1e-12
    np.testing.assert_allclose(res["imag_energies"], golden["ising_L10_D6_imag_dt005_energies"], rtol=1e-10, atol=0)
    assert abs(res["exc_E0"] - golden["ising_L10_D16_exc_E0"]) <= 1e-10 * abs(golden["ising_L10_D16_exc_E0"])
    assert abs(res["exc_E1"] - golden["ising_L10_D16_exc_E1"]) <= 1e-10 * abs(golden["ising_L10_D16_exc_E1"])
    t = mo.truncate_mps(mo.random_mps(10, 2, 16, 21), 5)
    big = mo.random_mps(10, 2, 16, 21)
    assert res["trunc_bond"] == 5
    assert abs(res["trunc_overlap"] - mo.contract_overlap(t, big).real) < 1e-10 * abs(res["trunc_overlap"])
    assert abs(res["trunc_norm"] - mo.contract_overlap(t, t).real) < 1e-10 * res["trunc_norm"]
    p = mo.product_mps(16, 2, 1)
    e = mo.contract_op(p, mo.schwinger_hmpo(16, 2.5, 100.0), p).real
    assert abs(res["schwinger_product_energy"] - e) < 1e-10 * abs(e)
