"""GPU test of mpsgpu_qr_device_noalloc, the QR entry point that allocates
nothing (its working memory is a fixed device array inside the library).

It is meant for callers that cannot allocate device memory when they need a
gauge move: a serving process whose allocator owns the whole HBM, or a loop
that must not fail on an allocation half way through a sweep.  The test
calls it twice in a row through the C ABI on device buffers (allocated here
by the test with torch) and checks both results against the allocating entry
point mpsgpu_qr, within the tolerance of the other QR tests.  It lives in a
file collected last, and passes alone in a fresh process as well.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run_noalloc(torch, capi, A):
    m, n = A.shape
    K = min(m, n)
    a = torch.from_numpy(np.asfortranarray(A).ravel(order="F").view(np.float64).copy()).cuda()
    q = torch.zeros(2 * m * K, dtype=torch.float64, device="cuda")
    r = torch.zeros(2 * K * n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    capi.qr_device_noalloc(m, n, a.data_ptr(), q.data_ptr(), r.data_ptr(), stream)
    torch.cuda.synchronize()
    Q = q.cpu().numpy().view(np.complex128).reshape(m, K, order="F")
    R = r.cpu().numpy().view(np.complex128).reshape(K, n, order="F")
    return Q, R


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
            scale = np.abs(A).max()
            assert np.abs(Qn - Qa).max() <= 1e-11 * max(1.0, np.abs(Qa).max())
            assert np.abs(Rn - Ra).max() <= 1e-11 * scale
            assert np.abs(Qn @ Rn - A).max() < 1e-13 * scale * max(m, n) ** 0.5


def test_noalloc_qr_rejects_oversize():
    pytest.importorskip("torch")
    from mpsdyn_b200 import capi

    with pytest.raises(capi.MpsgpuError) as ei:
        capi.qr_device_noalloc(1024, 512, 1, 1, 1, 0)  # never dereferenced: rejected first
    assert ei.value.status == 1
