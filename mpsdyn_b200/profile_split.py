"""One split-precision complex GEMM on the tensor cores, for profilers.

    python -m mpsdyn_b200.profile_split [--m 4096] [--n 4096] [--k 2048] [--repeats 0]

Builds seeded complex Gaussian A (m x k) and B (k x n) on the host, runs
C = A B once through mpsgpu_zgemm_split (operand preparation, then the
tcgen05 kernel), optionally times `--repeats` more runs with CUDA events, and
prints one JSON line with the times and the largest entrywise error relative
to |A||B| (checked against numpy on a 64 x 64 corner).
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from mpsdyn_b200 import capi


def main() -> None:
    p = argparse.ArgumentParser()
    p.add_argument("--m", type=int, default=4096)
    p.add_argument("--n", type=int, default=4096)
    p.add_argument("--k", type=int, default=2048)
    p.add_argument("--repeats", type=int, default=0)
    a = p.parse_args()
    rng = np.random.default_rng(0)
    A = rng.standard_normal((a.m, a.k)) + 1j * rng.standard_normal((a.m, a.k))
    B = rng.standard_normal((a.k, a.n)) + 1j * rng.standard_normal((a.k, a.n))
    with capi.Context(0) as ctx:
        C, t_all, t_mma = capi.zgemm_split(ctx, A, B, repeats=a.repeats)
    c = min(64, a.m, a.n)
    ref = A[:c] @ B[:, :c]
    rel = float(np.max(np.abs(C[:c, :c] - ref) / (np.abs(A[:c]) @ np.abs(B[:, :c]))))
    out = {"m": a.m, "n": a.n, "k": a.k, "max_rel_error_corner": rel}
    if a.repeats:
        fl = 8.0 * a.m * a.n * a.k
        out.update(ms_total=t_all, ms_mma=t_mma, bf16_tflops_mma=6 * fl / (t_mma * 1e-3) / 1e12,
                   fp64_equivalent_tflops_mma=fl / (t_mma * 1e-3) / 1e12)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
