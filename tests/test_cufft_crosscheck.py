"""Cross-check of the register FFT passes against cuFFT (through torch.fft on
the same GPU): the filtered horizontal derivatives of grad_velocity_filt
(compute_derivatives.f90:94-137) at production transform lengths.

cuFFT is the checker here, never the product: the library's transforms are
its own kernels.  Tolerances as for the oracle: 1e-12 (FP64), 1e-5 (mixed,
FP32 fields; cuFFT in complex64 on the same FP32 inputs)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _expected(f, lx, ly, dtype):
    """dfdx, dfdy and the Nyquist-filtered f by cuFFT (unnormalised forward
    scaled by 1/(nx ny), as the reference does; inverse unnormalised)."""
    import torch

    L, ny, nx = f.shape
    t = torch.as_tensor(f, device="cuda", dtype=dtype)
    F = torch.fft.rfft2(t)  # sum f e^{-i}: nx*ny times the reference's f_hat
    F[..., :, nx // 2] = 0  # kx Nyquist column
    F[..., ny // 2, :] = 0  # ky Nyquist row
    rdt = torch.float64 if dtype == torch.float64 else torch.float32
    kx = torch.arange(nx // 2 + 1, device="cuda", dtype=rdt) * (2 * math.pi / lx)
    kx[nx // 2] = 0
    j = torch.arange(ny, device="cuda")
    ky = (((j + ny // 2) % ny) - ny // 2).to(rdt) * (2 * math.pi / ly)
    ky[ny // 2] = 0
    dfdx = torch.fft.irfft2(1j * kx[None, None, :] * F, s=(ny, nx))
    dfdy = torch.fft.irfft2(1j * ky[None, :, None] * F, s=(ny, nx))
    ff = torch.fft.irfft2(F, s=(ny, nx))
    return [a.double().cpu().numpy() for a in (ff, dfdx, dfdy)]


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-5)])
@pytest.mark.parametrize("n", [64, 256, 512])
def test_grad_matches_cufft(gpu, n, precision, tol):
    import torch

    from new_repo_b200 import LES, RunParams

    p = RunParams(nx=n, ny=n, nz=2, dt=1e-4)
    les = LES(p, precision=precision)
    rng = np.random.default_rng(7)
    f = rng.standard_normal((p.nz + 2, p.ny, p.nx)) + 5.0
    if precision == "mixed":
        f = f.astype(np.float32).astype(np.float64)
    les.upload("u", f)
    les.grad_velocity_filt("u", "dudx", "dudy")
    got = [les.download(n_) for n_ in ("u", "dudx", "dudy")]
    want = _expected(f, p.lx, p.ly, torch.float64 if precision == "fp64" else torch.float32)
    for name, g, w in zip(("f", "dfdx", "dfdy"), got, want):
        e = _rel(g, w)
        assert e <= tol, (n, precision, name, e)
    les.close()
