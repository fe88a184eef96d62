"""Allocation-free horizontal derivatives (les_grad_xy_noalloc) against the
FP64 oracle and the solver entry point les_grad_velocity_filt on the same
fields, two calls in a row.  Tolerance: FP64 parity bar, max|a - b| / max|b|
<= 1e-12 per output.

Shapes: a square-free case, an x length with a radix-3 factor (96), and at
128x128 the largest level count whose spectra still fit the static buffer
(the last spectrum ends at the buffer's edge); one case runs on a stream the
caller created.
"""
import ctypes as C

import numpy as np
import pytest

SCRATCH = 32 << 20  # LES_NOALLOC_SCRATCH_BYTES


def _lib():
    from new_repo_b200 import capi

    return capi, capi.load()


def _scratch_bytes(nx, ny, nlev):
    """Bytes of the static buffer a call uses: two wavenumber tables, two
    twiddle tables and three FP64 spectra, each rounded up to 256 bytes."""
    a = lambda b: (b + 255) // 256 * 256  # noqa: E731
    lhx = nx // 2 + 1
    return 2 * a(8 * ny * lhx) + a(16 * nx) + a(16 * ny) + 3 * a(16 * nlev * ny * lhx)


def _max_levels(nx, ny):
    n = 1
    while _scratch_bytes(nx, ny, n + 1) <= SCRATCH:
        n += 1
    return n


def test_noalloc_rejects_sizes_beyond_the_static_buffer():
    """The size checks run before any CUDA call, so they need no GPU; the
    pointers are never dereferenced."""
    capi, lib = _lib()
    fake = C.c_void_p(256)
    rc = lib.les_grad_xy_noalloc(fake, fake, fake, 768, 512, 64, 1.0, 1.0, None)
    assert rc == capi.LES_ERR_INVALID
    msg = lib.les_noalloc_last_error().decode()
    assert "needs" in msg and "LES_NOALLOC_SCRATCH_BYTES" in msg
    # one level past the largest that fits at 128x128
    n = _max_levels(128, 128)
    assert lib.les_grad_xy_noalloc(fake, fake, fake, 128, 128, n + 1, 1.0, 1.0, None) == capi.LES_ERR_INVALID
    assert "needs" in lib.les_noalloc_last_error().decode()
    rc = lib.les_grad_xy_noalloc(None, fake, fake, 64, 64, 8, 1.0, 1.0, None)
    assert rc == capi.LES_ERR_INVALID


@pytest.mark.parametrize("ny", [24, 768, 96, 20])
def test_noalloc_rejects_y_lengths_without_a_y_pass(ny):
    """ny must have an equal-length y pass (powers of two 16..512): checked
    before anything is queued, so no GPU is needed."""
    capi, lib = _lib()
    fake = C.c_void_p(256)
    rc = lib.les_grad_xy_noalloc(fake, fake, fake, 64, ny, 2, 1.0, 1.0, None)
    assert rc == capi.LES_ERR_INVALID
    assert "ny one of" in lib.les_noalloc_last_error().decode()


CASES = [(64, 32, 16, False), (96, 64, 8, False), (128, 128, None, False), (64, 32, 16, True)]


def _solver_supports(nx, ny):
    """The solver also pads nx, ny by 3/2; its grids are powers of two."""
    return all(n in (16, 32, 64, 128, 256, 512) for n in (nx, ny))


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,nlev,own_stream", CASES)
def test_noalloc_matches_grad_velocity_filt_twice(gpu, nx, ny, nlev, own_stream):
    """Against the FP64 oracle's grad_velocity_filt on every shape, and
    against the solver's les_grad_velocity_filt where the solver takes the
    grid (x lengths with a factor 3 have no solver: their 3/2 padding is not
    a supported length)."""
    import torch

    from oracle import les_oracle as O
    from new_repo_b200 import LES, RunParams

    capi, lib = _lib()
    if nlev is None:
        nlev = _max_levels(nx, ny)
        assert _scratch_bytes(nx, ny, nlev) > SCRATCH - 3 * 16 * ny * (nx // 2 + 1)
    op = O.Params(nx=nx, ny=ny, nz=nlev - 2)
    ops = O.Ops(op)
    les = None
    if _solver_supports(nx, ny):
        les = LES(RunParams(nx=nx, ny=ny, nz=nlev - 2, dt=1e-4, sgs_model="cst_Smag"), precision="fp64")
    L = nlev
    rng = np.random.default_rng(nx + ny + nlev)
    stream = torch.cuda.Stream() if own_stream else None
    handle = C.c_void_p(stream.cuda_stream) if own_stream else None
    for call in range(2):
        f = rng.standard_normal((L, ny, nx))
        fo, dxo, dyo = f.copy(), np.zeros_like(f), np.zeros_like(f)
        O.grad_velocity_filt(ops, fo, dxo, dyo)
        refs = [("oracle", [fo, dxo, dyo])]
        if les is not None:
            les.upload("u", f)
            les.grad_velocity_filt("u", "dudx", "dudy")
            refs.append(("solver", [les.download(n) for n in ("u", "dudx", "dudy")]))
        dev = [torch.from_numpy(f.copy()).cuda(), torch.full_like(torch.from_numpy(f), 7.0).cuda(),
               torch.full_like(torch.from_numpy(f), -7.0).cuda()]
        torch.cuda.synchronize()
        rc = lib.les_grad_xy_noalloc(*(C.c_void_p(t.data_ptr()) for t in dev), nx, ny, L, op.lx, op.ly, handle)
        assert rc == capi.LES_OK, lib.les_noalloc_last_error().decode()
        if own_stream:
            stream.synchronize()
        torch.cuda.synchronize()
        got = [t.cpu().numpy() for t in dev]
        for who, ref in refs:
            for name, a, r in zip(("filtered f", "dfdx", "dfdy"), got, ref):
                err = np.abs(a - r).max() / np.abs(r).max()
                assert err <= 1e-12, f"{nx}x{ny}x{nlev} call {call} vs {who}: {name} rel err {err:.2e}"
    if les is not None:
        les.close()
