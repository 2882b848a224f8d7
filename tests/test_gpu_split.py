"""Split-precision complex GEMM on the tcgen05 tensor cores (BF16 limbs,
FP32 accumulation in TMEM) against the FP64 product, entrywise relative to
|A||B| (the scale its rounding error is bounded by)."""
import numpy as np
import pytest

from mpsdyn_b200 import capi

pytestmark = pytest.mark.gpu

# Three BF16 limbs carry 24 bits of every entry; the tensor cores' FP32
# accumulation adds an error that grows with K (measured 2.2e-6 of |A||B| at
# K = 1024, 2.9e-6 at K = 2048).  Entrywise bound, stated here:
def rel_tol(k):
    return 1e-6 + 3e-9 * k


def _crandn(rng, *shape, scale=1.0):
    return scale * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))


@pytest.mark.parametrize("m,n,k", [
    (128, 128, 16),     # one tile, one k-step
    (200, 130, 70),     # ragged in every dimension
    (640, 256, 128),    # first GEMM of the D = 128 Schwinger matvec (split K)
    (256, 128, 640),    # last GEMM of the same matvec (split K)
    (1024, 1024, 1024), # 64 k-steps through the four-stage ring
    (1280, 1280, 256),  # 128-column tiles
    (2048, 4096, 72),   # 128 x 256 tiles (enough of them to fill the SMs), ragged K
    (8, 3, 5),          # smaller than one tile
])
def test_split_gemm_accuracy(ctx, m, n, k):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    A = _crandn(rng, m, k)
    B = _crandn(rng, k, n, scale=1e3)  # a scale far from 1 exercises the limb split
    C, _, _ = capi.zgemm_split(ctx, A, B)
    ref = A @ B
    scale = np.abs(A) @ np.abs(B)
    rel = np.abs(C - ref) / scale
    print(f"split gemm {m}x{n}x{k}: max rel {rel.max():.2e}, mean {rel.mean():.2e}")
    assert np.isfinite(C).all()
    assert rel.max() <= rel_tol(k), rel.max()


def test_split_gemm_small_entries_and_zero_columns(ctx):
    rng = np.random.default_rng(11)
    A = _crandn(rng, 130, 48, scale=1e-20)
    B = _crandn(rng, 48, 70)
    B[:, 5] = 0.0
    C, _, _ = capi.zgemm_split(ctx, A, B)
    ref = A @ B
    assert np.all(C[:, 5] == 0.0)
    rel = np.abs(C - ref) / (np.abs(A) @ np.abs(B) + 1e-300)
    rel[:, 5] = 0.0
    assert rel.max() <= rel_tol(48), rel.max()


def test_split_gemm_timing_reports(ctx):
    rng = np.random.default_rng(3)
    A = _crandn(rng, 512, 512)
    B = _crandn(rng, 512, 512)
    C, t_all, t_mma = capi.zgemm_split(ctx, A, B, repeats=3)
    assert t_all > 0 and t_mma > 0 and t_mma <= t_all * 1.5
