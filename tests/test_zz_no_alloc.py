"""GPU test of mpsgpu_qr_device_noalloc, the QR entry point that allocates
nothing (its working memory is a fixed device array inside the library).

It is meant for callers that cannot allocate device memory when they need a
gauge move: a serving process whose allocator owns the whole HBM, or a loop
that must not fail on an allocation half way through a sweep.  The test
calls it twice in a row through the C ABI on device buffers (allocated here
by the test with torch) and checks both results against the allocating entry
point mpsgpu_qr, within the tolerance of the other QR tests; it also checks
the Q-only and R-only forms, a wide matrix, and that a call after the first
leaves the device's free memory unchanged.  It lives in a file collected
last, and passes alone in a fresh process as well.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _to_dev(torch, A):
    return torch.from_numpy(np.asfortranarray(A).ravel(order="F").view(np.float64).copy()).cuda()


def _run_noalloc(torch, capi, A, want_q=True, want_r=True):
    m, n = A.shape
    K = min(m, n)
    a = _to_dev(torch, A)
    q = torch.zeros(2 * m * K, dtype=torch.float64, device="cuda")
    r = torch.zeros(2 * K * n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    capi.qr_device_noalloc(m, n, a.data_ptr(), q.data_ptr() if want_q else 0, r.data_ptr() if want_r else 0,
                           stream)
    torch.cuda.synchronize()
    Q = q.cpu().numpy().view(np.complex128).reshape(m, K, order="F")
    R = r.cpu().numpy().view(np.complex128).reshape(K, n, order="F")
    return Q, R


def _check(A, Qa, Ra, Qn, Rn, q=True, r=True):
    m, n = A.shape
    scale = np.abs(A).max()
    if q:
        assert np.abs(Qn - Qa).max() <= 1e-11 * max(1.0, np.abs(Qa).max())
    if r:
        assert np.abs(Rn - Ra).max() <= 1e-11 * scale
    if q and r:
        assert np.abs(Qn @ Rn - A).max() < 1e-13 * scale * max(m, n) ** 0.5


def test_noalloc_qr_matches_allocating_qr_twice():
    torch = pytest.importorskip("torch")
    from mpsdyn_b200 import capi

    assert torch.cuda.is_available()
    rng = np.random.default_rng(2024)
    with capi.Context(0) as ctx:
        for (m, n) in [(256, 128), (40, 20)]:  # two calls in a row, different shapes
            A = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
            Qa, Ra = ctx.qr(A)
            Qn, Rn = _run_noalloc(torch, capi, A)
            _check(A, Qa, Ra, Qn, Rn)


def test_noalloc_qr_wide_and_single_outputs():
    torch = pytest.importorskip("torch")
    from mpsdyn_b200 import capi

    rng = np.random.default_rng(7)
    with capi.Context(0) as ctx:
        A = rng.standard_normal((48, 160)) + 1j * rng.standard_normal((48, 160))  # wide: m < n
        Qa, Ra = ctx.qr(A)
        Qn, Rn = _run_noalloc(torch, capi, A)
        _check(A, Qa, Ra, Qn, Rn)
        B = rng.standard_normal((200, 96)) + 1j * rng.standard_normal((200, 96))
        Qb, Rb = ctx.qr(B)
        Qq, _ = _run_noalloc(torch, capi, B, want_r=False)  # Q only
        _check(B, Qb, Rb, Qq, None, r=False)
        _, Rr = _run_noalloc(torch, capi, B, want_q=False)  # R only
        _check(B, Qb, Rb, None, Rr, q=False)


def test_noalloc_qr_second_call_allocates_nothing():
    torch = pytest.importorskip("torch")
    from mpsdyn_b200 import capi

    rng = np.random.default_rng(11)
    m, n = 320, 192
    A = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    with capi.Context(0) as ctx:  # creating the context places the fixed array
        K = min(m, n)
        a = _to_dev(torch, A)
        q = torch.zeros(2 * m * K, dtype=torch.float64, device="cuda")
        r = torch.zeros(2 * K * n, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        capi.qr_device_noalloc(m, n, a.data_ptr(), q.data_ptr(), r.data_ptr(), stream)  # warm-up call
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        capi.qr_device_noalloc(m, n, a.data_ptr(), q.data_ptr(), r.data_ptr(), stream)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        assert free1 == free0
        Qa, Ra = ctx.qr(A)
        Qn = q.cpu().numpy().view(np.complex128).reshape(m, K, order="F")
        Rn = r.cpu().numpy().view(np.complex128).reshape(K, n, order="F")
        _check(A, Qa, Ra, Qn, Rn)


def test_noalloc_qr_rejects_oversize():
    pytest.importorskip("torch")
    from mpsdyn_b200 import capi

    with pytest.raises(capi.MpsgpuError) as ei:
        capi.qr_device_noalloc(1024, 512, 1, 1, 1, 0)  # never dereferenced: rejected first
    assert ei.value.status == 1
