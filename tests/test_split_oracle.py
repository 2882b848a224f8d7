"""The split-precision arithmetic of the tensor-core path, restated on the
CPU (oracle/split_oracle.py) with exact accumulation: the limb split and the
i + j <= 2 product carry an error far below what the GPU shows, which comes
from the tensor cores' FP32 accumulation (tests/test_gpu_split.py)."""
import numpy as np
import pytest

from oracle import split_oracle as so


def test_bf16_round_is_nearest_with_8_bits():
    rng = np.random.default_rng(0)
    x = rng.standard_normal(20000) * np.exp(rng.uniform(-30, 30, 20000))
    h = so.bf16_round(x)
    m, _ = np.frexp(h)
    assert np.all(m * 256 == np.round(m * 256))           # 8 significant bits
    _, e = np.frexp(x)
    assert np.all(np.abs(x - h) <= np.ldexp(1.0, e - 9))    # half an ulp of bf16 (ulp = 2^(e-8))
    # exactly representable values are kept
    np.testing.assert_array_equal(so.bf16_round(h), h)


def test_three_limbs_carry_24_bits():
    rng = np.random.default_rng(1)
    x = rng.standard_normal(50000) * np.exp(rng.uniform(-20, 20, 50000))
    h, m, l = so.split3(x)
    assert np.all(np.abs(x - h - m - l) <= 2.0 ** -25 * np.abs(x))
    assert np.all(np.abs(m) <= 2.0 ** -8 * np.abs(x) * 1.01)
    assert np.all(np.abs(l) <= 2.0 ** -16 * np.abs(x) * 1.01)


@pytest.mark.parametrize("m,n,k", [(64, 64, 16), (128, 96, 640)])
def test_split_product_truncation_error(m, n, k):
    rng = np.random.default_rng(m + n + k)
    A = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    B = 1e3 * (rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n)))
    C = so.split_product(A, B)
    rel = np.abs(C - A @ B) / (np.abs(A) @ np.abs(B))
    # the scheme's own error; the GPU bound (1e-6 + 3e-9 K) is 30x or more above it
    assert rel.max() <= 3e-8, rel.max()


def test_fp32_accumulation_error_and_k_chunks():
    """With the tensor cores' FP32 accumulation restated, the error of a
    product with K = 640 (the last contraction of the D = 128 Schwinger
    matvec) stays inside the bound the GPU tests state, 1e-6 + 3e-9 K of
    |A||B|, and cutting K into chunks of five k-steps whose partials are added
    in FP64 (as the grouped split products do) lowers it."""
    rng = np.random.default_rng(640)
    m, n, k = 96, 64, 640
    A = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    B = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
    ref = A @ B
    scale = np.abs(A) @ np.abs(B)
    whole = (np.abs(so.split_product_fp32(A, B) - ref) / scale).max()
    chunked = (np.abs(so.split_product_fp32(A, B, chunk_steps=5) - ref) / scale).max()
    assert whole <= 1e-6 + 3e-9 * k, whole
    assert chunked < whole, (chunked, whole)
    # and both far above the limb truncation alone (the FP32 sums dominate)
    exact = (np.abs(so.split_product(A, B) - ref) / scale).max()
    assert exact < chunked
