"""Known-answer tests that pin the FP64 oracle (no GPU needed).

The reference ships no tests or golden data, so the oracle is pinned by
analytic answers of each operator plus the golden fixtures recorded by
tests/golden/make_golden.py.
"""
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import les_oracle as O


def _grid(nx=32, ny=32, nz=8):
    p = O.Params(nx=nx, ny=ny, nz=nz)
    x = np.arange(p.nx) * p.dx
    y = np.arange(p.ny) * p.dy
    return p, O.Ops(p), x, y


def test_fft_conventions_match_direct_dft():
    """FFTW r2c/c2r semantics: unnormalised both ways (fft_engine.f90:65-78)."""
    rng = np.random.default_rng(1)
    f = rng.standard_normal((6, 8))
    F = O.fft2_r2c(f)
    j, i = np.meshgrid(np.arange(6), np.arange(8), indexing="ij")
    direct = np.array([[np.sum(f * np.exp(-2j * np.pi * (kx * i / 8 + ky * j / 6))) for kx in range(5)]
                       for ky in range(6)])
    assert np.allclose(F, direct, atol=1e-12)
    assert np.allclose(O.fft2_c2r(F, 8, 6), f * 48, atol=1e-12)


def test_wavenumbers_nyquist_zeroed():
    p, ops, _, _ = _grid(16, 8)
    assert np.all(ops.kkx[:, -1] == 0) and np.all(ops.kky[:, -1] == 0)
    assert np.all(ops.kkx[p.ny // 2, :] == 0) and np.all(ops.kky[p.ny // 2, :] == 0)
    assert ops.kkx[0, 3] == pytest.approx(3.0)  # lx = 2 pi
    assert ops.kky[p.ny - 1, 0] == pytest.approx(-1.0)


def test_single_mode_derivatives():
    p, ops, x, y = _grid()
    f = np.zeros((p.nz + 2, p.ny, p.nx))
    f[:] = np.sin(5 * x)[None, None, :] * np.cos(3 * y)[None, :, None]
    dfdx, dfdy = np.zeros_like(f), np.zeros_like(f)
    g = f.copy()
    O.grad_velocity_filt(ops, g, dfdx, dfdy)
    assert np.abs(dfdx - 5 * np.cos(5 * x)[None, None, :] * np.cos(3 * y)[None, :, None]).max() < 1e-12
    assert np.abs(dfdy + 3 * np.sin(5 * x)[None, None, :] * np.sin(3 * y)[None, :, None]).max() < 1e-12
    assert np.abs(g - f).max() < 1e-13


def test_nyquist_mode_is_filtered_out():
    """grad_velocity_filt kills the kx = nx/2 and ky = ny/2 modes of f itself."""
    p, ops, x, y = _grid()
    f = np.zeros((p.nz + 2, p.ny, p.nx))
    f[:] = np.cos(p.nx // 2 * x)[None, None, :] + np.cos(p.ny // 2 * y)[None, :, None] + 2.0
    dx, dy = np.zeros_like(f), np.zeros_like(f)
    O.grad_velocity_filt(ops, f, dx, dy)
    assert np.abs(f - 2.0).max() < 1e-13


def test_ddz_linear_profile():
    p, ops, _, _ = _grid()
    z = np.arange(p.nz + 2)[:, None, None] * p.dz + np.zeros((1, p.ny, p.nx))
    out = np.zeros_like(z)
    O.ddz_uv(p, out, 3.0 * z)
    assert np.allclose(out[1:], 3.0, atol=1e-12)
    out[:] = 0
    O.ddz_w(p, out, 3.0 * z)
    assert np.allclose(out[1:p.nz + 1], 3.0, atol=1e-12) and np.all(out[p.nz + 1] == 0)


def test_padded_product_is_alias_free():
    """3/2 rule (compute_convective_padd.f90:274-388): the product of two
    modes whose sum exceeds the grid's band is exactly the truncated product."""
    p, ops, x, y = _grid(32, 32, 4)
    ax, by = 12, 11  # 2*12 = 24 > 16 aliases on the base grid
    a = np.cos(ax * x)[None, None, :] * np.cos(by * y)[None, :, None] + np.zeros((3, p.ny, p.nx))
    c = 1.0 / (p.nx * p.ny)
    A = O.transpose_to_big(p, c * a)
    prod = O.dealias_padd(p, A * A * (1.0 / ((3 * p.nx // 2) * (3 * p.ny // 2))))
    # exact: cos^2(12x) cos^2(11y) = 1/4 (1 + cos 24x)(1 + cos 22y); 24, 22 >= 16 are cut
    assert np.abs(prod - 0.25).max() < 1e-13


def test_trunc_rule_indices():
    """2/3 rule of compute_convective_trunc.f90:257,277,316,336."""
    p, ops, x, y = _grid(32, 32, 4)
    tt = math.ceil(32 / 3.0)  # keep modes 0..tt-2 = 0..9
    f = (np.cos(9 * x)[None, None, :] + np.cos(10 * x)[None, None, :]) + np.zeros((3, p.ny, p.nx))
    g = O.transpose_to_truncate(p, f / (p.nx * p.ny))
    assert tt == 11
    assert np.abs(g - np.cos(9 * x)[None, None, :]).max() < 1e-13
    tt2 = math.ceil(2 * p.lhy / 3.0)  # products: keep 0..10
    h = O.dealias_trunc(p, (f + np.cos(11 * x)[None, None, :]) / (p.nx * p.ny))
    assert tt2 == 12
    assert np.abs(h - f).max() < 1e-12


def test_test_filter_transfer_function():
    """Sharp cutoff kc = pi / (alpha sqrt(dx dy)) (testfilter.f90:101-131)."""
    p, ops, x, y = _grid(32, 32, 4)
    for alpha, G in ((2.0, ops.g_test), (4.0, ops.g_test_test)):
        kc = math.pi / (alpha * math.sqrt(p.dx * p.dy))
        for k in (2, 3, 5, 7, 9):
            f = np.cos(k * x)[None, None, :] + np.zeros((p.nz + 2, p.ny, p.nx))
            g = f.copy()
            O.test_filter(ops, g, G)
            expect = f if k * k < kc * kc else 0 * f
            assert np.abs(g[1:] - expect[1:]).max() < 1e-13, (alpha, k)


def test_tridiagonal_matches_dense_solve():
    p, ops, _, _ = _grid(16, 16, 6)
    rng = np.random.default_rng(3)
    r = rng.standard_normal((p.nz + 2, p.ny, p.lhx)) + 1j * rng.standard_normal((p.nz + 2, p.ny, p.lhx))
    r[0, 0, 0] = 0
    x = O.tridiag_solver_parallel(ops, r)
    a, b, c = O.tridiag_coeffs(ops)
    n = p.nz + 2
    for (j, i) in ((0, 0), (1, 2), (5, 3), (p.ny - 1, 1)):
        A = np.zeros((n, n))
        for k in range(n):
            A[k, k] = b[k, j, i]
            if k > 0:
                A[k, k - 1] = a[k, j, i]
            if k < n - 1:
                A[k, k + 1] = c[k, j, i]
        assert np.allclose(A @ x[:, j, i], r[:, j, i], atol=1e-10), (j, i)
    assert np.all(x[:, :, p.lhx - 1] == 0) and np.all(x[:, p.ny // 2, :] == 0)


def test_projection_makes_velocity_divergence_free():
    p = O.Params(nx=32, ny=32, nz=16)
    ops = O.Ops(p)
    st = O.make_state(p)
    d = O.les_step(ops, st)
    d = O.les_step(ops, st)
    # divergence of the projected field, measured with the next step's gradients
    O.compute_vel_grad(ops, st)
    div = st.dudx[1:p.nz + 1] + st.dvdy[1:p.nz + 1] + st.dwdz[1:p.nz + 1]
    assert np.sqrt((div ** 2).mean()) < 1e-10


def test_lasd_float_clips():
    """max(real(1E-24), real(x)) rounds to REAL(4) (compute_LagScaleDep.f90:624-690)."""
    x = np.array([0.1, 1e-30, -5.0, 1.0 + 1e-12])
    y = O.f32max_tiny(x)
    assert y[0] == float(np.float32(0.1))
    assert y[1] == float(np.float32(1e-24)) and y[2] == float(np.float32(1e-24))
    assert y[3] == 1.0


def test_lag_halo_reference_1x1_mirror_copy():
    """update_halo3 on a 1x1 process grid: low y halo holds rows 1, 2; high y
    halo rows ny-1, ny; x is wrapped periodically (decomp_2d_custom.f90:942-1024)."""
    p = O.Params(nx=8, ny=8, nz=4)
    F = np.zeros((p.nz + 2, p.ny, p.nx))
    F[1:] = np.arange(np.prod(F[1:].shape), dtype=float).reshape(F[1:].shape)
    FF = O.lag_halo(p, F)
    o = 1
    k = 2
    assert FF[k + o, 0 + o, 3 + o] == F[k, 1, 2]   # FF(3, 0, k) = F(3, 2, k)
    assert FF[k + o, 9 + o, 3 + o] == F[k, 6, 2]   # FF(3, ny+1, k) = F(3, ny-1, k)
    assert FF[k + o, 4 + o, 0 + o] == F[k, 3, 7]   # x wrap FF(0, 4, k) = F(nx, 4, k)
    assert FF[0 + o, 4 + o, 4 + o] == F[1, 3, 3]   # FF(:, :, 0) = FF(:, :, 1)
    assert FF[p.nz + 1 + o, 4 + o, 4 + o] == F[p.nz + 1, 3, 3]
    assert FF[p.nz + 1 + o, 4 + o, 0 + o] == F[p.nz - 1, 3, 7]  # top halo from level nz-1
    q = p.with_(lag_halo="periodic")
    GG = O.lag_halo(q, F)
    assert GG[k + o, 0 + o, 3 + o] == F[k, 7, 2]
    assert GG[p.nz + 1 + o, 4 + o, 0 + o] == F[p.nz + 1, 3, 7]


def test_les_step_is_deterministic():
    p = O.Params(nx=16, ny=16, nz=8)
    ops = O.Ops(p)
    a, b = O.make_state(p, seed=3), O.make_state(p, seed=3)
    for _ in range(6):
        O.les_step(ops, a)
        O.les_step(ops, b)
    assert np.array_equal(a.u, b.u) and np.array_equal(a.cs_opt2, b.cs_opt2)


GOLDEN = Path(__file__).parent / "golden"


@pytest.mark.parametrize("name", sorted(p.stem for p in GOLDEN.glob("*.npz")))
def test_golden_fixtures(name):
    """The oracle still reproduces the committed fixtures bit for bit (to 1e-13)."""
    from tests.golden.make_golden import CASES, run_case

    data = np.load(GOLDEN / f"{name}.npz")
    out = run_case(CASES[name])
    for k in data.files:
        ref = data[k]
        got = out[k]
        den = max(np.abs(ref).max(), 1e-300)
        assert np.abs(got - ref).max() / den < 1e-13, (name, k)
