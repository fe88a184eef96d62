"""Allocation-free horizontal derivatives (les_grad_xy_noalloc) against the
solver entry point les_grad_velocity_filt on the same fields, two calls in a
row.  Tolerance: FP64 parity bar, max|a - b| / max|b| <= 1e-12 per output
(the two paths run the same kernels; only the twiddle tables are computed on
a different processor).
"""
import ctypes as C

import numpy as np
import pytest


def _lib():
    from new_repo_b200 import capi

    return capi, capi.load()


def test_noalloc_rejects_sizes_beyond_the_static_buffer():
    """The size check runs before any CUDA call, so it needs no GPU; the
    pointers are never dereferenced."""
    capi, lib = _lib()
    fake = C.c_void_p(256)
    rc = lib.les_grad_xy_noalloc(fake, fake, fake, 768, 768, 64, 1.0, 1.0, None)
    assert rc == capi.LES_ERR_INVALID
    msg = lib.les_noalloc_last_error().decode()
    assert "needs" in msg and "LES_NOALLOC_SCRATCH_BYTES" in msg
    rc = lib.les_grad_xy_noalloc(None, fake, fake, 64, 64, 8, 1.0, 1.0, None)
    assert rc == capi.LES_ERR_INVALID


@pytest.mark.gpu
def test_noalloc_matches_grad_velocity_filt_twice(gpu):
    import torch

    from new_repo_b200 import LES, RunParams

    capi, lib = _lib()
    p = RunParams(nx=64, ny=32, nz=14, dt=1e-4, sgs_model="cst_Smag")
    les = LES(p, precision="fp64")
    L = p.nz + 2
    rng = np.random.default_rng(0)
    for call in range(2):
        f = rng.standard_normal((L, p.ny, p.nx))
        les.upload("u", f)
        les.grad_velocity_filt("u", "dudx", "dudy")
        ref = [les.download(n) for n in ("u", "dudx", "dudy")]
        dev = [torch.from_numpy(f.copy()).cuda(), torch.full_like(torch.from_numpy(f), 7.0).cuda(),
               torch.full_like(torch.from_numpy(f), -7.0).cuda()]
        torch.cuda.synchronize()
        rc = lib.les_grad_xy_noalloc(*(C.c_void_p(t.data_ptr()) for t in dev), p.nx, p.ny, L, p.lx, p.ly, None)
        assert rc == capi.LES_OK, lib.les_noalloc_last_error().decode()
        torch.cuda.synchronize()
        for name, t, r in zip(("filtered f", "dfdx", "dfdy"), dev, ref):
            a = t.cpu().numpy()
            err = np.abs(a - r).max() / np.abs(r).max()
            assert err <= 1e-12, f"call {call}: {name} rel err {err:.2e}"
    les.close()
