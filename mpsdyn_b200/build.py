"""Build libmpsgpu.so in-tree for sm_100a with nvcc (no JIT, no torch extension).

    python -m mpsdyn_b200.build        # or: python mpsdyn_b200/build.py

Objects go to mpsdyn_b200/_build/, the shared library to
mpsdyn_b200/libmpsgpu.so (found by mpsdyn_b200.capi).  The C++ facade with
the reference's class names (mpsdyn_b200/cpp) is built next to it as
mpsdyn_b200/libmpsdyn_facade.so (g++, links libmpsgpu.so, rpath $ORIGIN).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmpsgpu.so")
FACADE_DIR = os.path.join(HERE, "cpp")
FACADE_INC = os.path.join(FACADE_DIR, "include")
FACADE_LIB = os.path.join(HERE, "libmpsdyn_facade.so")

SOURCES = ["zgemm.cu", "blas1.cu", "lzstep.cu", "heff.cu", "qr.cu", "svd.cu", "grouped.cu", "umma.cu", "engine.cu", "capi.cu", "mpsio.cpp", "models.cpp", "server.cpp"]
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = [
    "-std=c++17", "-O3",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-Xcompiler", "-fPIC",
    "-Xptxas", "-warn-spills",
    "-diag-suppress", "177",
    "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
]


def _compile(src: str) -> str:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    srcp = os.path.join(CSRC, src)
    deps = [srcp] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "mpsgpu.h"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    cmd = [NVCC, *FLAGS, "-c", srcp, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    out = "\n".join(l for l in (r.stdout + r.stderr).splitlines() if "compute_100a" not in l or "error" in l)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{out}")
    if out.strip():
        print(out, file=sys.stderr)
    return obj


def build(verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(_compile, SOURCES))
    if not (os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(o) for o in objs)):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
        if verbose:
            print("built", LIB)
    build_facade(verbose)
    return LIB


def build_facade(verbose: bool = False) -> str:
    src = os.path.join(FACADE_DIR, "facade.cpp")
    deps = [src, LIB, os.path.join(ROOT, "include", "mpsgpu.h")] + [
        os.path.join(FACADE_INC, h) for h in os.listdir(FACADE_INC)]
    if os.path.exists(FACADE_LIB) and os.path.getmtime(FACADE_LIB) >= max(os.path.getmtime(d) for d in deps):
        return FACADE_LIB
    cmd = [os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall",
           "-I" + FACADE_INC, "-I" + os.path.join(ROOT, "include"), src, "-o", FACADE_LIB,
           "-L" + HERE, "-lmpsgpu", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("facade build failed:\n" + r.stdout + r.stderr)
    if verbose:
        print("built", FACADE_LIB)
    return FACADE_LIB


if __name__ == "__main__":
    build(verbose=True)
