"""CPU restatement of the split-precision complex product -- TEST
INFRASTRUCTURE ONLY (imported by ``tests/`` alone; the library never calls it).

The reference has no counterpart: it multiplies in complex FP64 through zgemm
(wrapper/wrapper.cpp).  The library's split-precision path (the tcgen05 GEMM
of ``mpsdyn_b200/csrc/umma.cu``) writes every FP64 real as three BF16 limbs,

    x = h + m + l,   h = bf16(x),  m = bf16(x - h),  l = bf16(x - h - m),

and keeps the limb products of combined order i + j <= 2 (the splitting of a
floating-point number into lower-precision terms whose products are summed,
as in Ootomo and Yokota's recovery of FP32 accuracy on FP16 tensor cores,
2022).  This module restates that arithmetic with exact (FP64) accumulation,
so the error it shows is the scheme's own truncation error; the tensor
cores' FP32 accumulation adds to it on the GPU.
"""
from __future__ import annotations

import numpy as np

BF16_BITS = 8  # significant bits of bfloat16, the implicit one included


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round FP64 values to the nearest bfloat16 value (ties to even), kept in
    FP64; normal range only (the limbs of the test data never leave it)."""
    x = np.asarray(x, dtype=np.float64)
    m, e = np.frexp(x)  # x = m 2^e, 0.5 <= |m| < 1
    r = np.round(m * 2.0 ** BF16_BITS) / 2.0 ** BF16_BITS  # np.round: half to even
    return np.ldexp(r, e)


def split3(x: np.ndarray):
    """The three limbs (h, m, l) of every entry of the real array x."""
    h = bf16_round(x)
    r1 = x - h
    m = bf16_round(r1)
    r2 = r1 - m
    return h, m, bf16_round(r2)


def split_product(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """C = A B (complex) from the limb products with i + j <= 2, summed
    exactly in FP64: Re C = sum ReA_i ReB_j - ImA_i ImB_j,
    Im C = sum ReA_i ImB_j + ImA_i ReB_j."""
    ar, ai = split3(A.real), split3(A.imag)
    br, bi = split3(B.real), split3(B.imag)
    cr = np.zeros((A.shape[0], B.shape[1]))
    ci = np.zeros_like(cr)
    for i in range(3):
        for j in range(3 - i):
            cr += ar[i] @ br[j] - ai[i] @ bi[j]
            ci += ar[i] @ bi[j] + ai[i] @ br[j]
    return cr + 1j * ci


def split_product_fp32(A: np.ndarray, B: np.ndarray, chunk_steps: int = 0) -> np.ndarray:
    """C = A B from the same limb products, accumulated as the tensor cores do:
    every MMA (one limb pair of one real product over a k-step of 16) adds its
    exact sum, rounded to FP32, into an FP32 accumulator.  With chunk_steps > 0
    the K range is cut into chunks of that many k-steps, each accumulated from
    zero in FP32, and the chunks' partial products are added in FP64 (the K
    chunks of the library's grouped split products).  Emulation of the
    rounding, not of the hardware's internal order inside one MMA."""
    m, k = A.shape
    n = B.shape[1]
    ar, ai = split3(A.real), split3(A.imag)
    br, bi = split3(B.real), split3(B.imag)
    ksteps = (k + 15) // 16
    per = chunk_steps if chunk_steps > 0 else ksteps
    f32 = np.float32
    out_r = np.zeros((m, n))
    out_i = np.zeros((m, n))
    for c0 in range(0, ksteps, per):
        acc_r = np.zeros((m, n), dtype=f32)
        acc_i = np.zeros((m, n), dtype=f32)
        for t in range(c0, min(ksteps, c0 + per)):
            s = slice(16 * t, min(k, 16 * t + 16))
            for i in range(3):
                for j in range(3 - i):
                    acc_r = (acc_r + (ar[i][:, s] @ br[j][s, :]).astype(f32)).astype(f32)
                    acc_r = (acc_r - (ai[i][:, s] @ bi[j][s, :]).astype(f32)).astype(f32)
                    acc_i = (acc_i + (ar[i][:, s] @ bi[j][s, :]).astype(f32)).astype(f32)
                    acc_i = (acc_i + (ai[i][:, s] @ br[j][s, :]).astype(f32)).astype(f32)
        out_r += acc_r.astype(np.float64)
        out_i += acc_i.astype(np.float64)
    return out_r + 1j * out_i
