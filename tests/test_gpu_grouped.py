"""GPU parity of the grouped matvec (many instances of different shapes in
one grouped launch sequence, optionally replayed from a CUDA graph) against
the oracle's TensorMultiplier::product restatement; complex FP64, relative
error <= 1e-13 of max |y| per instance."""
import numpy as np
import pytest

from oracle import mps_oracle as mo

pytestmark = pytest.mark.gpu


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a.ravel(order="F"))).cuda()


def test_grouped_matvec_matches_oracle(ctx):
    torch = pytest.importorskip("torch")
    from mpsdyn_b200 import capi
    rng = np.random.default_rng(7)
    shapes = [(2, 3, 3, 32, 32), (2, 5, 5, 64, 64), (2, 3, 3, 7, 9), (2, 5, 5, 130, 96), (3, 4, 4, 20, 18),
              (2, 3, 3, 1, 4), (2, 5, 5, 256, 256)]
    keep, inst, refs = [], [], []
    for (d, wl, Dl, Dr) in [(s[0], s[1], s[3], s[4]) for s in shapes]:
        wr = wl
        c = lambda *sh: rng.standard_normal(sh) + 1j * rng.standard_normal(sh)
        L, W, R, x = c(Dl, wl, Dl), c(d, wl, d, wr), c(Dr, wr, Dr), c(d, Dl, Dr)
        refs.append(mo.heff_apply(L, W, R, x))                  # (d, Dl, Dr)
        tL, tW = _dev(torch, L), _dev(torch, W)
        tR = _dev(torch, R.transpose(2, 1, 0))                  # (ket, w, bra)
        tx = _dev(torch, x.transpose(1, 0, 2))                  # (Dl, d, Dr)
        ty = torch.zeros(d * Dl * Dr, dtype=torch.complex128, device="cuda")
        keep += [tL, tW, tR, tx, ty]
        inst.append(dict(d=d, wl=wl, wr=wr, Dl=Dl, Dr=Dr, L=tL.data_ptr(), W=tW.data_ptr(), Rt=tR.data_ptr(),
                         x=tx.data_ptr(), y=ty.data_ptr()))
    for repeats in (0, 3):
        ms, fl = capi.heff_matvec_grouped(ctx, inst, repeats)
        torch.cuda.synchronize()
        for k, (ref, s) in enumerate(zip(refs, inst)):
            y = keep[5 * k + 4].cpu().numpy().reshape(s["Dl"], s["d"], s["Dr"], order="F").transpose(1, 0, 2)
            err = np.abs(y - ref).max() / np.abs(ref).max()
            assert err < 1e-13, (k, err)
        assert fl > 0
        if repeats:
            assert ms is not None and ms > 0


# Split precision (BF16 limbs on the tcgen05 tensor cores, FP32 accumulation):
# the accumulation error grows about linearly with the inner dimension K of
# the larger GEMM (measured: 3.6e-5 of max |y| at D = 512, w = 5, K = 2560);
# bound per instance, relative to max |y|, stated here:
def split_tol(k):
    return 2e-6 + 4e-8 * k


def test_grouped_matvec_split_precision(ctx):
    torch = pytest.importorskip("torch")
    from mpsdyn_b200 import capi
    rng = np.random.default_rng(8)
    shapes = [(2, 5, 5, 256, 256), (2, 3, 3, 130, 96), (2, 5, 5, 64, 64), (3, 4, 4, 20, 18), (2, 3, 3, 1, 4),
              (2, 5, 5, 512, 512)]
    keep, inst, refs = [], [], []
    for (d, wl, wr, Dl, Dr) in shapes:
        c = lambda *sh: rng.standard_normal(sh) + 1j * rng.standard_normal(sh)
        L, W, R, x = c(Dl, wl, Dl), c(d, wl, d, wr), c(Dr, wr, Dr), c(d, Dl, Dr)
        refs.append(mo.heff_apply(L, W, R, x))
        tL, tW = _dev(torch, L), _dev(torch, W)
        tR = _dev(torch, R.transpose(2, 1, 0))
        tx = _dev(torch, x.transpose(1, 0, 2))
        ty = torch.zeros(d * Dl * Dr, dtype=torch.complex128, device="cuda")
        keep += [tL, tW, tR, tx, ty]
        inst.append(dict(d=d, wl=wl, wr=wr, Dl=Dl, Dr=Dr, L=tL.data_ptr(), W=tW.data_ptr(), Rt=tR.data_ptr(),
                         x=tx.data_ptr(), y=ty.data_ptr()))
    for repeats in (0, 2):
        ms, fl, mp = capi.heff_matvec_grouped_ex(ctx, inst, 1, repeats)
        torch.cuda.synchronize()
        errs = []
        for k, (ref, s) in enumerate(zip(refs, inst)):
            y = keep[5 * k + 4].cpu().numpy().reshape(s["Dl"], s["d"], s["Dr"], order="F").transpose(1, 0, 2)
            errs.append(np.abs(y - ref).max() / np.abs(ref).max())
        print("split grouped errors", ["%.1e" % e for e in errs])
        for e, s in zip(errs, inst):
            assert e <= split_tol(max(s["Dl"], s["Dr"] * s["wr"])), errs
        assert fl > 0 and mp > 0
        if repeats:
            assert ms is not None and ms > 0
