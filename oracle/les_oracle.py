"""CPU FP64 oracle for the LES time step -- TEST INFRASTRUCTURE ONLY.

This module restates, routine by routine, the single-rank behaviour of the
Fortran pseudo-spectral ABL LES (fmargairaz/new-repo, ``src/*.f90``).  It is
the checker for the CUDA library in ``new_repo_b200``: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may
import it, and never as the thing measured or shipped.

Parity status: **parity unpinned**.  The reference is Fortran + MPI + FFTW +
2DECOMP&FFT, none of which can be built here, and it ships no golden vectors
or tests.  This restatement is pinned instead by analytic known-answer tests
(single-mode spectral derivatives, exact padded products of band-limited
fields, the tridiagonal solve against a dense solve, filter transfer
functions) in ``tests/test_oracle.py``, and by the golden fixtures that
``tests/golden/make_golden.py`` records from it.

Conventions
-----------
* Every 3-D field is a C-ordered ``numpy`` array of shape ``(nz+2, ny, nx)``
  indexed ``[k, j, i]`` with ``k`` the Fortran level (0 .. nz+1, ghosts at 0
  and nz+1), ``j = j_f - 1`` and ``i = i_f - 1``.  This is byte-for-byte the
  Fortran ``(nx, ny, 0:nz+1)`` layout.  Fields the reference dimensions
  ``(nx, ny, nz+1)`` (levels 1..nz+1) or ``(nx, ny, nz)`` use the same shape
  with the unused levels left alone.
* Spectral planes are ``[.., ky, kx]`` with ``kx = 0 .. nx/2`` -- the FFTW
  r2c half-spectrum ``(lhx, ny)`` of ``decomp_2d_fft_2d.f90``.
* FFTs are unnormalised in both directions, as FFTW's are
  (``fft_engine.f90:65-78``); callers pre-scale by ``1/(nx*ny)``.
* The third-party arithmetic boundary is FFTW 3.x (version unpinned in
  ``src/Makefile:63,83``); it is replaced here by scipy's pocketfft, which
  computes the same unnormalised DFTs (the c2r inverse ignores the imaginary
  part of the kx=0 and kx=nx/2 bins, as FFTW's does).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np
import scipy.fft as sfft

# parameters_IO.f90:42-49
PI = 3.1415926535897932384626433
KVONK = 0.4
BOGUS = -1.23456789e20

# compute_LagScaleDep.f90:27-29
TF1, TF1_2 = 2.0, 4.0
TF2, TF2_2 = 4.0, 16.0
OPFTIME = 1.5
F32_TINY = np.float32(1e-24)  # the default-real literal 1E-24

WORKERS = 1  # scipy.fft worker threads (bench's CPU leg raises this)


def set_workers(n: int) -> None:
    global WORKERS
    WORKERS = max(1, int(n))


@dataclass
class Params:
    """Mirror of the namelist-derived globals of ``parameters_IO.f90``.

    ``read_parameters`` (parameters_IO.f90:238-264) non-dimensionalises the
    namelist; ``derive()`` repeats that arithmetic in the same order.
    """

    nx: int = 32
    ny: int = 32
    nz: int = 32
    dt: float = 2e-4
    # physical_param (dimensional, before derive())
    xy_pi: bool = True
    lx_in: float = 2.0
    ly_in: float = 2.0
    lz_in: float = 1.0
    zi: float = 1.0
    u_scale: float = 1.0
    lbc_dz0: float = 1e-4
    pfx: float = 1.0
    pfy: float = 0.0
    re: float = 5e4
    # sgs_param
    cs0: float = 0.16
    sgs_model: str = "dyn_LagScaleDep"  # 'cst_Smag' | 'dyn_Smag' | 'dyn_LagScaleDep'
    cs_count: int = 5
    dyn_init: int = 5
    # momentum_bc
    lbc_special: str = "wall_law"
    wall_model: str = "wall_filter"  # 'wall_filter' | 'wall_inst' | 'wall_homog'
    # build option -DDEA_PADD / -DDEA_TRUNC (src/Makefile:16-26)
    dealias: str = "padd"
    # Halo of the Lagrangian interpolation (decomp_2d_custom.f90:902-1024).
    # 'reference1x1' reproduces what update_halo3 yields on a 1x1 process
    # grid (self-messages with equal tags: mirror copies, see lag_halo()).
    # 'periodic' is the decomposition-independent periodic wrap.
    lag_halo: str = "reference1x1"

    # derived
    lx: float = field(init=False, default=0.0)
    ly: float = field(init=False, default=0.0)
    lz: float = field(init=False, default=0.0)
    dx: float = field(init=False, default=0.0)
    dy: float = field(init=False, default=0.0)
    dz: float = field(init=False, default=0.0)
    z0: float = field(init=False, default=0.0)

    def __post_init__(self):
        self.derive()

    def derive(self) -> "Params":
        lx, ly, lz = self.lx_in, self.ly_in, self.lz_in
        if self.xy_pi:  # parameters_IO.f90:243-245
            lx = lx * PI
            ly = ly * PI
        lx = lx / self.zi  # :248
        ly = ly / self.zi
        lz = lz / self.zi
        self.lx, self.ly, self.lz = lx, ly, lz
        self.dx = lx / float(self.nx)  # :275-277
        self.dy = ly / float(self.ny)
        self.dz = lz / float(self.nz)
        self.z0 = self.lbc_dz0 / self.zi  # boundary_condition_mpi.f90:126
        return self

    @property
    def lhx(self) -> int:
        return self.nx // 2 + 1

    @property
    def lhy(self) -> int:
        return self.ny // 2 + 1

    def with_(self, **kw) -> "Params":
        q = replace(self, **kw)
        return q.derive()


# ---------------------------------------------------------------------------
# spectral runtime (fft_engine.f90, decomp_2d_fft_2d.f90)
# ---------------------------------------------------------------------------
def build_wavenumbers(p: Params):
    """fft_engine.f90:97-145 -- kkx, kky, kk2 on the (ky, kx) half-plane with
    the Nyquist row and column set to zero."""
    nx, ny, lhx, lhy = p.nx, p.ny, p.lhx, p.lhy
    kkx = np.zeros((ny, lhx))
    kky = np.zeros((ny, lhx))
    for i in range(lhx):
        kkx[:, i] = float(i)
    for j in range(ny):
        kky[j, :] = float(((j + ny // 2) % ny) - ny // 2)
    kkx[:, lhx - 1] = 0.0
    kky[:, lhx - 1] = 0.0
    kkx[lhy - 1, :] = 0.0
    kky[lhy - 1, :] = 0.0
    kkx = 2.0 * PI / p.lx * kkx
    kky = 2.0 * PI / p.ly * kky
    kk2 = kkx * kkx + kky * kky
    return kkx, kky, kk2


def fft2_r2c(f):
    """fft_2d_r2c (decomp_2d_fft_2d.f90:498-532): x r2c then y c2c, unnormalised."""
    return sfft.rfft2(f, axes=(-2, -1), workers=WORKERS)


def fft2_c2r(fh, nx, ny):
    """fft_2d_c2r (decomp_2d_fft_2d.f90:546-577): y c2c then x c2r, unnormalised."""
    return sfft.irfft2(fh, s=(ny, nx), axes=(-2, -1), norm="forward", workers=WORKERS)


def kill_oddballs(fh, p: Params):
    """Zero the kx=nx/2 column and the ky=ny/2 row (compute_derivatives.f90:105-119)."""
    fh[..., :, p.lhx - 1] = 0.0
    fh[..., p.lhy - 1, :] = 0.0
    return fh


def test_filter_create(p: Params, alpha: float, kk2):
    """testfilter.f90:101-131 -- sharp cutoff kernel including 1/(nx*ny).

    ``where (real(kk2) >= kc2)`` compares kk2 rounded to default REAL(4)."""
    g = np.full((p.ny, p.lhx), 1.0 / (p.nx * p.ny))
    delta = alpha * math.sqrt(p.dx * p.dy)
    kc2 = (PI / delta) ** 2
    g[kk2.astype(np.float32).astype(np.float64) >= kc2] = 0.0
    g[:, p.lhx - 1] = 0.0
    g[p.ny // 2, :] = 0.0
    return g


class Ops:
    """Per-grid constants shared by the operators (wavenumbers, filter kernels)."""

    def __init__(self, p: Params):
        self.p = p
        self.kkx, self.kky, self.kk2 = build_wavenumbers(p)
        self.g_test = test_filter_create(p, 2.0, self.kk2)  # LES_engine.f90:152
        self.g_test_test = test_filter_create(p, 4.0, self.kk2)  # :153
        self.delta = (p.dx * p.dy * p.dz) ** (1.0 / 3.0)  # compute_sgs.f90:144
        # compute_dynamic_coeff exponent log(tf1)/(log(tf2)-log(tf1))
        self.beta_pow = math.log(TF1) / (math.log(TF2) - math.log(TF1))


# ---------------------------------------------------------------------------
# compute_derivatives.f90
# ---------------------------------------------------------------------------
def grad_velocity_filt(ops: Ops, f, dfdx, dfdy):
    """compute_derivatives.f90:94-137 -- spectral d/dx, d/dy on all levels
    0..nz+1; f is overwritten by its Nyquist-filtered self."""
    p = ops.p
    const = 1.0 / (p.nx * p.ny)
    fh = kill_oddballs(fft2_r2c(const * f), p)
    ikx = 1j * ops.kkx * fh
    iky = 1j * ops.kky * fh
    dfdx[:] = fft2_c2r(ikx, p.nx, p.ny)
    dfdy[:] = fft2_c2r(iky, p.nx, p.ny)
    f[:] = fft2_c2r(fh, p.nx, p.ny)


def ddz_uv(p: Params, dfdz, f):
    """compute_derivatives.f90:375-400 -- uvp -> w nodes, k = 1..nz+1."""
    const = 1.0 / p.dz
    dfdz[1:] = const * (f[1:] - f[:-1])


def ddz_w(p: Params, dfdz, f):
    """compute_derivatives.f90:413-441 -- w -> uvp nodes, k = 1..nz; top level 0."""
    const = 1.0 / p.dz
    nz = p.nz
    dfdz[1:nz + 1] = const * (f[2:nz + 2] - f[1:nz + 1])
    dfdz[nz + 1] = 0.0


def div_stress(ops: Ops, rhs, tx, ty, tz, stag, want_layers=False):
    """compute_derivatives.f90:464-577 -- rhs(1..nz) += dx tx + dy ty + dz tz.

    Returns (bottom_wk_press, top_wk_press) for the w equation (stag=False)."""
    p = ops.p
    nz = p.nz
    const = 1.0 / (p.nx * p.ny)
    fh = kill_oddballs(fft2_r2c(const * tx), p)
    dtxdx = fft2_c2r(1j * ops.kkx * fh, p.nx, p.ny)
    fh = kill_oddballs(fft2_r2c(const * ty), p)
    dtydy = fft2_c2r(1j * ops.kky * fh, p.nx, p.ny)
    dtzdz = np.zeros_like(tz)
    if stag:
        ddz_w(p, dtzdz, tz)
    else:
        ddz_uv(p, dtzdz, tz)
    rhs[1:nz + 1] = rhs[1:nz + 1] + dtxdx[1:nz + 1] + dtydy[1:nz + 1] + dtzdz[1:nz + 1]
    if want_layers:
        if not stag:
            bottom = dtxdx[1] + dtydy[1] + dtzdz[1]
            top = dtxdx[nz + 1] + dtydy[nz + 1]
        else:
            bottom = np.full((p.ny, p.nx), BOGUS)
            top = np.full((p.ny, p.nx), BOGUS)
        return bottom, top
    return None


# ---------------------------------------------------------------------------
# boundary_condition_mpi.f90
# ---------------------------------------------------------------------------
def set_bc(p: Params, pos, var, bc_type, bc, stag):
    """boundary_condition_mpi.f90:33-63."""
    nz = p.nz
    if pos == "bot":
        if stag:
            if bc_type == "drc":
                var[0] = 2.0 * bc - var[1]
            elif bc_type == "neu":
                var[0] = var[1] - bc * p.dz
        else:
            if bc_type == "drc":
                var[1] = bc
    else:
        if stag:
            if bc_type == "drc":
                var[nz + 1] = 2.0 * bc - var[nz]
            elif bc_type == "neu":
                var[nz + 1] = var[nz] + bc * p.dz
        else:
            if bc_type == "drc":
                var[nz + 1] = bc


# ---------------------------------------------------------------------------
# compute_wall_law.f90 (+ utility_tools.f90 layer filter, testfilter.f90)
# ---------------------------------------------------------------------------
def test_filter_layer(f2d, g):
    """testfilter.f90:197-210 -- 2-D cutoff filter of one plane (G holds 1/(nx*ny))."""
    ny, nx = f2d.shape
    return fft2_c2r(g * fft2_r2c(f2d), nx, ny)


def wall_layer(ops: Ops, st: "State"):
    """u1, v1, u_avg of obukhov/wallstress (compute_wall_law.f90:119-151, 210-243)."""
    p = ops.p
    if p.wall_model == "wall_filter":
        u1 = test_filter_layer(st.u[1].copy(), ops.g_test)
        v1 = test_filter_layer(st.v[1].copy(), ops.g_test)
    elif p.wall_model == "wall_inst":
        u1 = st.u[1].copy()
        v1 = st.v[1].copy()
    elif p.wall_model == "wall_homog":  # utility_tools.f90:140-168
        const = 1.0 / (p.nx * p.ny)
        u1 = np.full((p.ny, p.nx), const * st.u[1].sum())
        v1 = np.full((p.ny, p.nx), const * st.v[1].sum())
    else:
        raise ValueError("Invalid wall law type")
    u_avg = np.sqrt(u1 ** 2 + v1 ** 2)
    return u1, v1, u_avg


def obukhov(ops: Ops, st: "State"):
    """compute_wall_law.f90:198-254 (neutral): u* = kappa*U/ln(dz/2/z0)."""
    p = ops.p
    _, _, u_avg = wall_layer(ops, st)
    st.u_star_avg[:] = KVONK * u_avg / np.log((0.5 * p.dz) / st.lbc_z0)


def wallstress(ops: Ops, st: "State"):
    """compute_wall_law.f90:107-185 -- Neumann ghost value and wall stress at k=1."""
    p = ops.p
    u1, v1, u_avg = wall_layer(ops, st)
    zero = u_avg == 0.0
    nz_ = ~zero
    with np.errstate(divide="ignore", invalid="ignore"):
        bc_u = st.u_star_avg / (0.5 * p.dz * KVONK) * u1 / u_avg
        bc_v = st.u_star_avg / (0.5 * p.dz * KVONK) * v1 / u_avg
        txz1 = (st.u_star_avg ** 2) * u1 / u_avg
        tyz1 = (st.u_star_avg ** 2) * v1 / u_avg
    st.lbc_u[:] = np.where(nz_, bc_u, 0.0)
    st.lbc_v[:] = np.where(nz_, bc_v, 0.0)
    st.dudz[1] = st.lbc_u
    st.dvdz[1] = st.lbc_v
    st.txz[1] = np.where(nz_, txz1, 0.0)
    st.tyz[1] = np.where(nz_, tyz1, 0.0)


# ---------------------------------------------------------------------------
# compute_sgs.f90
# ---------------------------------------------------------------------------
def compute_sij(p: Params, st: "State"):
    """compute_sgs.f90:260-335 -- S_ij on uvp at k=1, on w nodes for k=2..nz+1.

    Returns six arrays shaped like a field (levels 1..nz+1 valid)."""
    nz = p.nz
    shp = st.u.shape
    s11, s12, s13, s22, s23, s33 = (np.zeros(shp) for _ in range(6))
    ux = st.dudx[1]
    uy = st.dudy[1]
    if p.lbc_special == "wall_law":
        uz = st.dudz[1]
        vz = st.dvdz[1]
    else:
        uz = 0.5 * (st.dudz[1] + st.dudz[2])
        vz = 0.5 * (st.dvdz[1] + st.dvdz[2])
    vx = st.dvdx[1]
    vy = st.dvdy[1]
    wx = 0.5 * (st.dwdx[1] + st.dwdx[2])
    wy = 0.5 * (st.dwdy[1] + st.dwdy[2])
    wz = st.dwdz[1]
    s11[1] = ux
    s12[1] = 0.5 * (uy + vx)
    s13[1] = 0.5 * (uz + wx)
    s22[1] = vy
    s23[1] = 0.5 * (vz + wy)
    s33[1] = wz
    k = slice(2, nz + 2)
    km = slice(1, nz + 1)
    ux = 0.5 * (st.dudx[k] + st.dudx[km])
    uy = 0.5 * (st.dudy[k] + st.dudy[km])
    uz = st.dudz[k]
    vx = 0.5 * (st.dvdx[k] + st.dvdx[km])
    vy = 0.5 * (st.dvdy[k] + st.dvdy[km])
    vz = st.dvdz[k]
    wx = st.dwdx[k]
    wy = st.dwdy[k]
    wz = 0.5 * (st.dwdz[k] + st.dwdz[km])
    s11[k] = ux
    s12[k] = 0.5 * (uy + vx)
    s13[k] = 0.5 * (uz + wx)
    s22[k] = vy
    s23[k] = 0.5 * (vz + wy)
    s33[k] = wz
    return s11, s12, s13, s22, s23, s33


def strain_norm(s11, s12, s13, s22, s23, s33):
    """|S| = sqrt(2 S_ij S_ij) (compute_sgs.f90:181-182, compute_LagScaleDep.f90:243-244)."""
    return np.sqrt(2.0 * (s11 ** 2 + s22 ** 2 + s33 ** 2 + 2.0 * (s12 ** 2 + s13 ** 2 + s23 ** 2)))


def sgs_stress(ops: Ops, st: "State", jt: int, jtt: int):
    """compute_sgs.f90:105-247 (LES branch)."""
    p = ops.p
    nz = p.nz
    delta = ops.delta
    lvec = np.full(nz + 2, delta)
    s11, s12, s13, s22, s23, s33 = compute_sij(p, st)
    if p.sgs_model == "cst_Smag":
        n_dmp = 2.0
        z = 0.5 * p.dz
        lvec[1] = (p.cs0 ** n_dmp * (KVONK * z) ** (-n_dmp) + delta ** (-n_dmp)) ** (-1.0 / n_dmp)
        for k in range(2, nz + 2):
            z = (1 + k - 2.0) * p.dz
            lvec[k] = (p.cs0 ** n_dmp * (KVONK * z) ** (-n_dmp) + delta ** (-n_dmp)) ** (-1.0 / n_dmp)
        st.cs_opt2[1:] = p.cs0 ** 2
    elif p.sgs_model == "dyn_LagScaleDep":
        lasd_coeff(ops, st, s11, s12, s22, s33, s13, s23, jt, jtt)
    elif p.sgs_model == "dyn_Smag":
        dynsmag_coeff(ops, st, s11, s12, s22, s33, s13, s23, jt, jtt)
    else:
        raise ValueError("Invalid SGS model")
    k = slice(1, nz + 2)
    stmp = strain_norm(s11[k], s12[k], s13[k], s22[k], s23[k], s33[k])
    st.nu_t[k] = stmp * st.cs_opt2[k] * (lvec[1:nz + 2] ** 2)[:, None, None]
    nu = st.nu_t
    # bottom layer on uvp nodes (:195-203)
    st.txx[1] = 2.0 * nu[1] * st.dudx[1]
    st.txy[1] = 2.0 * nu[1] * 0.5 * (st.dudy[1] + st.dvdx[1])
    st.tyy[1] = 2.0 * nu[1] * st.dvdy[1]
    st.tzz[1] = 2.0 * nu[1] * st.dwdz[1]
    k = slice(2, nz + 1)
    kp = slice(3, nz + 2)
    const = 0.5 * (nu[k] + nu[kp])
    st.txx[k] = 2.0 * const * st.dudx[k]
    st.txy[k] = 2.0 * const * 0.5 * (st.dudy[k] + st.dvdx[k])
    st.tyy[k] = 2.0 * const * st.dvdy[k]
    st.tzz[k] = 2.0 * const * st.dwdz[k]
    k = slice(2, nz + 2)
    st.txz[k] = 2.0 * nu[k] * s13[k]
    st.tyz[k] = 2.0 * nu[k] * s23[k]
    st.tzz[0] = st.tzz[1]
    return s11, s12, s13, s22, s23, s33


# ---------------------------------------------------------------------------
# testfilter.f90 (3-D) and compute_LagScaleDep.f90
# ---------------------------------------------------------------------------
def test_filter(ops: Ops, f, g):
    """testfilter.f90:144-184 -- filter levels 1..nz+1 in place."""
    p = ops.p
    f[1:] = fft2_c2r(fft2_r2c(f[1:]) * g, p.nx, p.ny)


def f32(x):
    """Fortran ``real(x)`` with no kind: round to default REAL(4)."""
    return np.asarray(x, dtype=np.float64).astype(np.float32)


def f32max_tiny(x):
    """``max(real(1E-24), real(x))`` promoted back to real(8)."""
    return np.maximum(F32_TINY, f32(x)).astype(np.float64)


def dynamic_mum(ops: Ops, st: "State", S, s11, s12, s22, s33, s13, s23, tf_2, g):
    """compute_LagScaleDep.f90:485-596 -- AB = L:M and BB = M:M at one test scale
    (levels 1..nz+1).  Returns AB, BB as field-shaped arrays."""
    p = ops.p
    nz = p.nz
    const = 2.0 * ops.delta ** 2
    shp = st.u.shape
    u_ft, v_ft, w_ft = np.zeros(shp), np.zeros(shp), np.zeros(shp)
    u_ft[1] = st.u[1]
    v_ft[1] = st.v[1]
    w_ft[1] = 0.25 * st.w[2]
    k = slice(2, nz + 2)
    km = slice(1, nz + 1)
    u_ft[k] = 0.5 * (st.u[k] + st.u[km])
    v_ft[k] = 0.5 * (st.v[k] + st.v[km])
    w_ft[k] = st.w[k]
    a11 = u_ft * u_ft
    a12 = u_ft * v_ft
    a13 = u_ft * w_ft
    a23 = v_ft * w_ft
    a22 = v_ft * v_ft
    a33 = w_ft * w_ft
    for f in (u_ft, v_ft, w_ft):
        test_filter(ops, f, g)
    for a, (x, y) in ((a11, (u_ft, u_ft)), (a12, (u_ft, v_ft)), (a13, (u_ft, w_ft)),
                      (a22, (v_ft, v_ft)), (a23, (v_ft, w_ft)), (a33, (w_ft, w_ft))):
        test_filter(ops, a, g)
        a -= x * y
    sf = [s.copy() for s in (s11, s12, s13, s22, s23, s33)]
    for s in sf:
        test_filter(ops, s, g)
    s11f, s12f, s13f, s22f, s23f, s33f = sf
    s_ft = np.sqrt(2.0 * (s11f ** 2 + s22f ** 2 + s33f ** 2 + 2.0 * (s12f ** 2 + s13f ** 2 + s23f ** 2)))
    ss = [S * s for s in (s11, s12, s13, s22, s23, s33)]
    for s in ss:
        test_filter(ops, s, g)
    ss11, ss12, ss13, ss22, ss23, ss33 = ss
    b11 = const * (ss11 - tf_2 * s_ft * s11f)
    b12 = const * (ss12 - tf_2 * s_ft * s12f)
    b13 = const * (ss13 - tf_2 * s_ft * s13f)
    b22 = const * (ss22 - tf_2 * s_ft * s22f)
    b23 = const * (ss23 - tf_2 * s_ft * s23f)
    b33 = const * (ss33 - tf_2 * s_ft * s33f)
    ab = a11 * b11 + a22 * b22 + a33 * b33 + 2.0 * (a12 * b12 + a13 * b13 + a23 * b23)
    bb = b11 ** 2 + b22 ** 2 + b33 ** 2 + 2.0 * (b12 ** 2 + b13 ** 2 + b23 ** 2)
    return ab, bb


def lag_halo(p: Params, F):
    """FF of compute_interpolag_coeff (compute_LagScaleDep.f90:439-452) built as
    update_halo3(F, FF, 2, dcp) (decomp_2d_custom.f90:902-1024) leaves it.

    Returns FF indexed [k+1, j+1, i+1] for Fortran k in -1..nz+2,
    j in -1..ny+2, i in -1..nx+2 (F levels 1..nz+1 in F[1:nz+2]).

    On a 1x1 process grid every halo message is a self-message with tag 0, so
    MPI's in-order matching pairs the first receive with the first send: the
    low halo receives the first two interior rows/planes and the high halo
    the last two (a mirror copy, not a periodic wrap).  x is always wrapped
    locally (:942-955)."""
    nx, ny, nz = p.nx, p.ny, p.nz
    FF = np.full((nz + 4, ny + 4, nx + 4), np.nan)
    o = 1  # array index = Fortran index + o
    FF[1 + o:nz + 1 + o, 1 + o:ny + 1 + o, 1 + o:nx + 1 + o] = F[1:nz + 1]
    # x wrap on levels 1..nz, rows 1..ny
    FF[1 + o:nz + 1 + o, 1 + o:ny + 1 + o, -1 + o:1 + o] = F[1:nz + 1, :, nx - 2:nx]
    FF[1 + o:nz + 1 + o, 1 + o:ny + 1 + o, nx + 1 + o:nx + 3 + o] = F[1:nz + 1, :, 0:2]
    if p.lag_halo == "reference1x1":
        FF[:, -1 + o:1 + o, :] = FF[:, 1 + o:3 + o, :]
        FF[:, ny + 1 + o:ny + 3 + o, :] = FF[:, ny - 1 + o:ny + 1 + o, :]
        FF[-1 + o:1 + o] = FF[1 + o:3 + o]
        FF[nz + 1 + o:nz + 3 + o] = FF[nz - 1 + o:nz + 1 + o]
    elif p.lag_halo == "periodic":
        FF[:, -1 + o:1 + o, :] = FF[:, ny - 1 + o:ny + 1 + o, :]
        FF[:, ny + 1 + o:ny + 3 + o, :] = FF[:, 1 + o:3 + o, :]
        # the top level's halos wrap the top level itself
        top = np.empty((ny + 4, nx + 4))
        top[1 + o:ny + 1 + o, 1 + o:nx + 1 + o] = F[nz + 1]
        top[1 + o:ny + 1 + o, -1 + o:1 + o] = F[nz + 1, :, nx - 2:nx]
        top[1 + o:ny + 1 + o, nx + 1 + o:nx + 3 + o] = F[nz + 1, :, 0:2]
        top[-1 + o:1 + o] = top[ny - 1 + o:ny + 1 + o]
        top[ny + 1 + o:ny + 3 + o] = top[1 + o:3 + o]
        FF[nz + 1 + o] = top
        FF[nz + 2 + o] = top
    else:
        raise ValueError(p.lag_halo)
    # compute_LagScaleDep.f90:441-452
    FF[0 + o] = FF[1 + o]
    FF[-1 + o] = BOGUS
    FF[nz + 1 + o, 1 + o:ny + 1 + o, 1 + o:nx + 1 + o] = F[nz + 1]
    FF[nz + 2 + o, 1 + o:ny + 1 + o, 1 + o:nx + 1 + o] = F[nz + 1]
    return FF


def interpolag_weight(p: Params, st: "State"):
    """compute_LagScaleDep.f90:309-411 -- neighbour offsets and weights."""
    nz = p.nz
    cs = float(p.cs_count)
    tmp = st.u_lag / cs
    st.u_lag[1] = tmp[1]
    st.u_lag[2:nz + 2] = 0.5 * (tmp[2:nz + 2] + tmp[1:nz + 1])
    tmp = st.v_lag / cs
    st.v_lag[1] = tmp[1]
    st.v_lag[2:nz + 2] = 0.5 * (tmp[2:nz + 2] + tmp[1:nz + 1])
    st.w_lag[:] = st.w_lag / cs
    st.w_lag[1] = 0.25 * st.w_lag[2]
    k = slice(1, nz + 2)
    xp = -st.u_lag[k] * p.dt * cs / p.dx
    yp = -st.v_lag[k] * p.dt * cs / p.dy
    zp = -st.w_lag[k] * p.dt * cs / p.dz
    # first-cell correction (:368-379); note zp(:,:,1) is taken from zp(:,:,2)
    zp[1] = zp[1] + np.minimum(zp[1], 0.0)
    zp[0] = zp[0] + np.maximum(zp[0], 0.0)
    zp[1] = np.minimum(1.0, zp[1])
    zp[0] = np.minimum(1.0, zp[1])
    zp[1] = np.maximum(-1.0, zp[1])
    zp[0] = np.maximum(-1.0, zp[1])
    addx = np.where(np.signbit(xp), -1, 1)
    addy = np.where(np.signbit(yp), -1, 1)
    addz = np.where(np.signbit(zp), -1, 1)
    return addx, addy, addz, np.abs(xp), np.abs(yp), np.abs(zp)


def interpolag_coeff(p: Params, F, w):
    """compute_LagScaleDep.f90:427-474 -- trilinear upstream interpolation of F
    on levels 1..nz+1 (in place)."""
    nx, ny, nz = p.nx, p.ny, p.nz
    addx, addy, addz, cx, cy, cz = w
    FF = lag_halo(p, F)
    K, J, I = np.meshgrid(np.arange(1, nz + 2), np.arange(1, ny + 1), np.arange(1, nx + 1), indexing="ij")
    ax = I + addx
    ay = J + addy
    az = K + addz
    o = 1
    fx, fy, fz = 1.0 - cx, 1.0 - cy, 1.0 - cz

    def g(i, j, k):
        return FF[k + o, j + o, i + o]

    F[1:nz + 2] = (fx * fy * (g(I, J, K) * fz + g(I, J, az) * cz) + fx * cy * (g(I, ay, K) * fz + g(I, ay, az) * cz)
                   + cx * fy * (g(ax, J, K) * fz + g(ax, J, az) * cz) + cx * cy * (g(ax, ay, K) * fz + g(ax, ay, az) * cz))


def update_interpolag_coeff(p: Params, ops: Ops, F_AB, F_BB, AB, BB):
    """compute_LagScaleDep.f90:607-640 with the default-REAL casts of :624,626,633."""
    k = slice(1, p.nz + 2)
    powcoeff = -1.0 / 8.0
    opftdelta = OPFTIME * ops.delta
    lagran_dt = p.dt * float(p.cs_count)
    tmp = np.maximum(f32(F_AB[k] * F_BB[k]), F32_TINY).astype(np.float64)
    tmp = opftdelta * tmp ** powcoeff
    tmp = f32max_tiny(tmp)
    dumfac = lagran_dt / tmp
    epsi = dumfac / (1.0 + dumfac)
    F_AB[k] = epsi * AB[k] + (1.0 - epsi) * F_AB[k]
    F_BB[k] = epsi * BB[k] + (1.0 - epsi) * F_BB[k]
    F_AB[k] = f32max_tiny(F_AB[k])


def dynamic_coeff(p: Params, ops: Ops, st: "State"):
    """compute_LagScaleDep.f90:651-707 -- Cs^2 = Cs^2_2D / beta with the REAL(4) clips."""
    nz = p.nz
    k = slice(1, nz + 2)
    c2 = f32max_tiny(st.F_LM[k] / st.F_MM[k])
    c4 = f32max_tiny(st.F_QN[k] / st.F_NN[k])
    beta = (c4 / c2) ** ops.beta_pow
    beta = np.maximum(f32(beta), np.float32(1.0 / (TF1 * TF2))).astype(np.float64)
    beta[nz] = 1.0  # level nz+1
    st.beta[k] = beta
    st.cs_opt2[k] = f32max_tiny(c2 / beta)


def lasd_coeff(ops: Ops, st: "State", s11, s12, s22, s33, s13, s23, jt, jtt):
    """compute_LagScaleDep.f90:204-298."""
    p = ops.p
    nz = p.nz
    if jtt >= p.dyn_init:
        st.u_lag += st.u
        st.v_lag += st.v
        st.w_lag += st.w
    if jtt < p.dyn_init:
        st.cs_opt2[1:] = 0.03
    elif jtt % p.cs_count == 0:
        S = np.zeros_like(st.u)
        S[1:] = strain_norm(s11[1:], s12[1:], s13[1:], s22[1:], s23[1:], s33[1:])
        LM, MM = dynamic_mum(ops, st, S, s11, s12, s22, s33, s13, s23, TF1_2, ops.g_test)
        QN, NN = dynamic_mum(ops, st, S, s11, s12, s22, s33, s13, s23, TF2_2, ops.g_test_test)
        if st.f_coeff_init:
            w = interpolag_weight(p, st)
            for F in (st.F_LM, st.F_MM, st.F_QN, st.F_NN):
                interpolag_coeff(p, F, w)
        else:
            k = slice(1, nz + 2)
            st.F_MM[k] = MM[k]
            st.F_LM[k] = 0.03 * MM[k]
            st.F_NN[k] = NN[k]
            st.F_QN[k] = 0.03 * NN[k]
            st.f_coeff_init = True
        update_interpolag_coeff(p, ops, st.F_LM, st.F_MM, LM, MM)
        update_interpolag_coeff(p, ops, st.F_QN, st.F_NN, QN, NN)
        dynamic_coeff(p, ops, st)
        st.lagran_init = True
        st.u_lag[:] = 0.0
        st.v_lag[:] = 0.0
        st.w_lag[:] = 0.0


def dynsmag_coeff(ops: Ops, st: "State", s11, s12, s22, s33, s13, s23, jt, jtt):
    """compute_DynSmag.f90:61-245 -- plane-averaged Germano coefficient."""
    p = ops.p
    nz = p.nz
    if jtt < p.dyn_init:
        st.cs_opt2[1:] = 0.03
        return
    if jt % p.cs_count != 0:
        return
    S = np.zeros_like(st.u)
    S[1:] = strain_norm(s11[1:], s12[1:], s13[1:], s22[1:], s23[1:], s33[1:])
    LM, MM = dynamic_mum(ops, st, S, s11, s12, s22, s33, s13, s23, 4.0, ops.g_test)
    k = slice(1, nz + 2)
    num = LM[k].sum(axis=(1, 2)) / (p.nx * p.ny)
    den = MM[k].sum(axis=(1, 2)) / (p.nx * p.ny)
    cs_z = np.where(den != 0.0, num / np.where(den != 0.0, den, 1.0), 0.0)
    cs_z = np.maximum(0.0, cs_z)
    st.cs_opt2[k] = cs_z[:, None, None]


# ---------------------------------------------------------------------------
# compute_convective_padd.f90 / compute_convective_trunc.f90
# ---------------------------------------------------------------------------
def _r2c_x(f):
    return sfft.rfft(f, axis=-1, workers=WORKERS)


def _c2r_x(F, n):
    return sfft.irfft(F, n=n, axis=-1, norm="forward", workers=WORKERS)


def transpose_to_big(p: Params, cc):
    """compute_convective_padd.f90:274-324 -- separable 3/2 zero padding of
    levels 0..nz+1 (x pass, transpose, y pass)."""
    nx, ny, lhx, lhy = p.nx, p.ny, p.lhx, p.lhy
    nx2, ny2 = 3 * nx // 2, 3 * ny // 2
    scr = _r2c_x(cc)
    big = np.zeros(scr.shape[:-1] + (nx2 // 2 + 1,), dtype=complex)
    big[..., :lhx - 1] = scr[..., :lhx - 1]
    hyb = _c2r_x(big, nx2)  # (L, ny, nx2)
    hyb_t = np.swapaxes(hyb, -1, -2)  # y along last axis
    scr = _r2c_x(hyb_t)
    big = np.zeros(scr.shape[:-1] + (ny2 // 2 + 1,), dtype=complex)
    big[..., :lhy - 1] = scr[..., :lhy - 1]
    out = _c2r_x(big, ny2)  # (L, nx2, ny2)
    return np.ascontiguousarray(np.swapaxes(out, -1, -2))  # (L, ny2, nx2)


def dealias_padd(p: Params, cc_big):
    """compute_convective_padd.f90:337-388 -- truncate the fine-grid product back."""
    nx, ny, lhx, lhy = p.nx, p.ny, p.lhx, p.lhy
    t = np.swapaxes(cc_big, -1, -2)  # (L, nx2, ny2)
    scr_big = _r2c_x(t)
    scr = np.zeros(scr_big.shape[:-1] + (lhy,), dtype=complex)
    scr[..., :lhy - 1] = scr_big[..., :lhy - 1]
    hyb = _c2r_x(scr, ny)  # (L, nx2, ny)
    hyb = np.swapaxes(hyb, -1, -2)  # (L, ny, nx2)
    scr_big = _r2c_x(hyb)
    scr = np.zeros(scr_big.shape[:-1] + (lhx,), dtype=complex)
    scr[..., :lhx - 1] = scr_big[..., :lhx - 1]
    return _c2r_x(scr, nx)


def transpose_to_truncate(p: Params, cc):
    """compute_convective_trunc.f90:244-293 -- zero modes tt=ceil(n/3).. in x and y."""
    nx, ny = p.nx, p.ny
    scr = _r2c_x(cc)
    tt = math.ceil(float(nx) / 3.0)
    scr[..., tt - 1:] = 0.0
    wk = _c2r_x(scr, nx)
    wk = np.swapaxes(wk, -1, -2)
    scr = _r2c_x(wk)
    tt = math.ceil(float(ny) / 3.0)
    scr[..., tt - 1:] = 0.0
    out = _c2r_x(scr, ny)
    return np.ascontiguousarray(np.swapaxes(out, -1, -2))


def dealias_trunc(p: Params, cc):
    """compute_convective_trunc.f90:303-352 -- zero modes tt=ceil(2*lh/3).. ."""
    nx, ny, lhx, lhy = p.nx, p.ny, p.lhx, p.lhy
    t = np.swapaxes(cc, -1, -2)
    scr = _r2c_x(t)
    tt = math.ceil(float(2 * lhy) / 3.0)
    scr[..., tt - 1:] = 0.0
    wk = _c2r_x(scr, ny)
    wk = np.swapaxes(wk, -1, -2)
    scr = _r2c_x(wk)
    tt = math.ceil(float(2 * lhx) / 3.0)
    scr[..., tt - 1:] = 0.0
    return _c2r_x(scr, nx)


def compute_dealias_convec(p: Params, st: "State", cx, cy, cz):
    """compute_convective_padd.f90:115-262 (dealias='padd') or
    compute_convective_trunc.f90:115-235 (dealias='trunc'): rotational form u x omega."""
    nz = p.nz
    const = 1.0 / (p.nx * p.ny)
    cx[:] = -const * st.u
    cy[:] = -const * st.v
    cz[:] = -const * st.w
    to_big = transpose_to_big if p.dealias == "padd" else transpose_to_truncate
    ub, vb, wb = to_big(p, cx), to_big(p, cy), to_big(p, cz)
    cx[:] = const * (st.dwdy - st.dvdz)
    cy[:] = const * (st.dudz - st.dwdx)
    cz[:] = const * (st.dvdx - st.dudy)
    if p.lbc_special == "wall_law":
        cx[0] = 0.0
        cy[0] = 0.0
        cx[1] = const * (0.5 * (st.dwdy[1] + st.dwdy[2]) - st.dvdz[1])
        cy[1] = const * (st.dudz[1] - 0.5 * (st.dwdx[1] + st.dwdx[2]))
    o1, o2, o3 = to_big(p, cx), to_big(p, cy), to_big(p, cz)
    if p.dealias == "padd":
        c = 1.0 / ((3 * p.nx // 2) * (3 * p.ny // 2))
        back = dealias_padd
    else:
        c = 1.0 / (p.nx * p.ny)
        back = dealias_trunc
    wk = np.zeros_like(ub)
    k = slice(2, nz + 1)
    kp = slice(3, nz + 2)
    km = slice(1, nz)
    # x term (:184-204)
    wk[1] = c * (-vb[1] * o3[1] + 0.5 * wb[2] * o2[2])
    wk[k] = c * (-vb[k] * o3[k] + 0.5 * (wb[kp] * o2[kp] + wb[k] * o2[k]))
    cx[1:nz + 1] = back(p, wk[1:nz + 1])
    # y term (:208-227)
    wk[1] = c * (ub[1] * o3[1] + 0.5 * wb[2] * (-o1[2]))
    wk[k] = c * (ub[k] * o3[k] + 0.5 * (wb[k] * (-o1[k]) + wb[kp] * (-o1[kp])))
    cy[1:nz + 1] = back(p, wk[1:nz + 1])
    # z term (:231-249)
    wk[1] = 0.0
    wk[k] = c * 0.5 * ((ub[k] + ub[km]) * (-o2[k]) + (vb[k] + vb[km]) * (o1[k]))
    cz[1:nz + 1] = back(p, wk[1:nz + 1])
    if p.dealias == "padd":  # :251-259
        for f in (cx, cy, cz):
            f[0] = BOGUS
            f[nz + 1] = BOGUS


# ---------------------------------------------------------------------------
# compute_pressure.f90
# ---------------------------------------------------------------------------
def tridiag_coeffs(ops: Ops):
    """build_matrix (compute_pressure.f90:544-619): a, b, c of shape (nz+2, ny, lhx)
    (row index 0 = Fortran row 1)."""
    p = ops.p
    nz = p.nz
    shp = (nz + 2, p.ny, p.lhx)
    a = np.zeros(shp)
    b = np.zeros(shp)
    c = np.zeros(shp)
    a[0] = BOGUS
    b[0] = -1.0
    c[0] = 1.0
    a[nz + 1] = -1.0
    b[nz + 1] = 1.0
    c[nz + 1] = BOGUS
    a[1:nz + 1] = 1.0 / (p.dz ** 2)
    b[1:nz + 1] = -(ops.kkx ** 2 + ops.kky ** 2 + 2.0 / (p.dz ** 2))
    c[1:nz + 1] = 1.0 / (p.dz ** 2)
    a[0, 0, 0] = 0.0
    b[0, 0, 0] = 1.0
    c[0, 0, 0] = 0.0
    return a, b, c


def tridiag_solver_parallel(ops: Ops, r):
    """compute_pressure.f90:448-493 -- Thomas per (kx,ky); the Nyquist row and
    column are skipped (left at zero here; the caller zeroes them anyway)."""
    p = ops.p
    a, b, c = tridiag_coeffs(ops)
    n = p.nz + 2
    x = np.zeros_like(r)
    gam = np.zeros(r.shape, dtype=np.float64)
    bet = b[0].copy()
    with np.errstate(divide="ignore", invalid="ignore"):  # Nyquist columns are singular and skipped
        x[0] = r[0] / bet
        for k in range(1, n):
            gam[k] = c[k - 1] / bet
            bet = b[k] - a[k] * gam[k]
            x[k] = (r[k] - a[k] * x[k - 1]) / bet
        for k in range(n - 2, -1, -1):
            x[k] = x[k] - gam[k + 1] * x[k + 1]
    x[:, :, p.lhx - 1] = 0.0
    x[:, p.lhy - 1, :] = 0.0
    return x


def press_stag_array(ops: Ops, st: "State", tadv1: float):
    """compute_pressure.f90:116-242 (+ poisson_solver :256-305,
    compute_press_grad :320-372)."""
    p = ops.p
    nz = p.nz
    const = 1.0 / (p.nx * p.ny)
    rH = []
    for f in (st.u, st.v, st.w):
        r = np.zeros_like(f)
        r[1:nz + 1] = const / tadv1 * (f[1:nz + 1] / p.dt)
        rH.append(r)
    st.bottom_wk_press[:] = const * st.bottom_wk_press
    bot = fft2_r2c(st.bottom_wk_press)
    top = fft2_r2c(const * st.top_wk_press)
    Hx, Hy, Hz = (fft2_r2c(r) for r in rH)
    for H in (Hx, Hy, Hz):
        H[1:nz + 1, :, p.lhx - 1] = 0.0
        H[1:nz + 1, p.lhy - 1, :] = 0.0
    for L in (bot, top):
        L[:, p.lhx - 1] = 0.0
        L[p.lhy - 1, :] = 0.0
    bot = bot * p.dz
    top = top * p.dz
    wk = np.zeros((nz + 2, p.ny, p.lhx), dtype=complex)
    k = slice(1, nz + 1)
    kp = slice(2, nz + 2)
    wk[k] = 1j * (ops.kkx * Hx[k] + ops.kky * Hy[k]) + (Hz[kp] - Hz[k]) / p.dz
    # poisson_solver: rows 1 / 2..nz+1 / nz+2
    r = np.zeros((nz + 2, p.ny, p.lhx), dtype=complex)
    r[0] = bot
    r[1:nz + 1] = wk[1:nz + 1]
    r[nz + 1] = top
    r[0, 0, 0] = 0.0
    x = tridiag_solver_parallel(ops, r)
    wk[1:nz + 1] = x[1:nz + 1]
    wk[0] = x[0]  # gather_layer_spz
    wk[nz + 1] = 0.0
    wk[:, :, p.lhx - 1] = 0.0
    wk[:, p.lhy - 1, :] = 0.0
    # compute_press_grad
    st.dpdx[1:nz + 1] = fft2_c2r(1j * ops.kkx * wk[1:nz + 1], p.nx, p.ny)
    st.dpdy[1:nz + 1] = fft2_c2r(1j * ops.kky * wk[1:nz + 1], p.nx, p.ny)
    st.p[:] = fft2_c2r(wk, p.nx, p.ny)
    st.p[nz + 1] = BOGUS
    st.dpdz[1:nz + 1] = (1.0 / p.dz) * (st.p[1:nz + 1] - st.p[0:nz])


# ---------------------------------------------------------------------------
# state, initial conditions and the time step (LES_engine.f90)
# ---------------------------------------------------------------------------
FIELDS = ("u", "v", "w", "dudx", "dudy", "dudz", "dvdx", "dvdy", "dvdz", "dwdx", "dwdy", "dwdz",
          "p", "dpdx", "dpdy", "dpdz", "rhsx", "rhsy", "rhsz", "rhsx_f", "rhsy_f", "rhsz_f",
          "txx", "txy", "txz", "tyy", "tyz", "tzz", "cs_opt2", "nu_t",
          "F_LM", "F_MM", "F_QN", "F_NN", "beta", "u_lag", "v_lag", "w_lag")
PLANES = ("lbc_u", "lbc_v", "lbc_w", "ubc_u", "ubc_v", "ubc_w", "bottom_wk_press", "top_wk_press",
          "lbc_z0", "u_star_avg")


class State:
    """Global arrays of system.f90:21-43 plus the module-private SGS/wall state."""

    def __init__(self, p: Params):
        self.p = p
        shp = (p.nz + 2, p.ny, p.nx)
        for n in FIELDS:
            setattr(self, n, np.zeros(shp))
        for n in PLANES:
            setattr(self, n, np.zeros((p.ny, p.nx)))
        self.lbc_z0[:] = p.z0  # set_bc_surface (boundary_condition_mpi.f90:124-129)
        self.w[0] = BOGUS  # system.f90:196-198
        self.f_coeff_init = False
        self.lagran_init = False
        self.jt_total = 0
        # wall law switches the lower u,v BC to Neumann (LES_engine.f90:168-171)
        self.lbc_typ = {"u": "drc", "v": "drc", "w": "drc"}
        self.ubc_typ = {"u": "neu", "v": "neu", "w": "drc"}

    def copy(self) -> "State":
        s = State.__new__(State)
        s.__dict__.update({k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in self.__dict__.items()})
        s.lbc_typ = dict(self.lbc_typ)
        s.ubc_typ = dict(self.ubc_typ)
        return s


def rng_uniform(seed: int, field_id: int, shape):
    """Counter-based uniform noise in [-1, 1): splitmix64 of
    (seed, field, linear index).  Not the reference's ran3 generator."""
    n = int(np.prod(shape))
    x = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = x + np.uint64((seed * 1000003 + field_id * 7919 + 1) & 0xFFFFFFFFFFFFFFFF) * np.uint64(0x9E3779B97F4A7C15)
        z = x
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u01 = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return (2.0 * u01 - 1.0).reshape(shape)


def log_law_fields(p: Params, seed: int = 0, amp: float = 0.1):
    """Synthetic initial velocity (nz, ny, nx): u = ln(z/z0)/0.4 at uvp heights
    (initial_conditions.f90:101-117 with u_star=1, pfx>0) plus uniform noise."""
    z = (np.arange(1, p.nz + 1) - 0.5) * p.dz
    arg = (1.0 / KVONK) * np.log(z / p.z0)
    shape = (p.nz, p.ny, p.nx)
    u = np.broadcast_to(arg[:, None, None], shape).copy()
    v = np.zeros(shape)
    w = np.zeros(shape)
    u += amp * rng_uniform(seed, 0, shape)
    v += amp * rng_uniform(seed, 1, shape)
    w += amp * rng_uniform(seed, 2, shape)
    return u, v, w


def set_initial_conditions(p: Params, st: State, u, v, w):
    """The ic_type='files' path (initial_conditions.f90:130-165, 183-212):
    load (nz,ny,nx) fields, no noise, then the initial BCs (lbc still Dirichlet)."""
    nz = p.nz
    st.u[1:nz + 1] = u
    st.v[1:nz + 1] = v
    st.w[1:nz + 1] = w
    zero = np.zeros((p.ny, p.nx))
    set_bc(p, "bot", st.u, "drc", zero, True)
    set_bc(p, "bot", st.v, "drc", zero, True)
    set_bc(p, "bot", st.w, "drc", zero, False)
    set_bc(p, "top", st.u, "neu", zero, True)
    set_bc(p, "top", st.v, "neu", zero, True)
    set_bc(p, "top", st.w, "drc", zero, False)
    st.w[0] = BOGUS
    if p.lbc_special == "wall_law":
        st.lbc_typ["u"] = "neu"
        st.lbc_typ["v"] = "neu"


def compute_vel_grad(ops: Ops, st: State):
    """LES_engine.f90:449-498."""
    p = ops.p
    grad_velocity_filt(ops, st.u, st.dudx, st.dudy)
    grad_velocity_filt(ops, st.v, st.dvdx, st.dvdy)
    grad_velocity_filt(ops, st.w, st.dwdx, st.dwdy)
    apply_bcs(p, st)
    ddz_uv(p, st.dudz, st.u)
    ddz_uv(p, st.dvdz, st.v)
    ddz_w(p, st.dwdz, st.w)


def apply_bcs(p: Params, st: State):
    set_bc(p, "bot", st.u, st.lbc_typ["u"], st.lbc_u, True)
    set_bc(p, "bot", st.v, st.lbc_typ["v"], st.lbc_v, True)
    set_bc(p, "bot", st.w, st.lbc_typ["w"], st.lbc_w, False)
    set_bc(p, "top", st.u, st.ubc_typ["u"], st.ubc_u, True)
    set_bc(p, "top", st.v, st.ubc_typ["v"], st.ubc_v, True)
    set_bc(p, "top", st.w, st.ubc_typ["w"], st.ubc_w, False)


def compute_rhs_adv(ops: Ops, st: State):
    """LES_engine.f90:509-572."""
    p = ops.p
    nz = p.nz
    st.rhsx_f[1:nz + 1] = st.rhsx[1:nz + 1]
    st.rhsy_f[1:nz + 1] = st.rhsy[1:nz + 1]
    st.rhsz_f[1:nz + 1] = st.rhsz[1:nz + 1]
    st.rhsx[1:nz + 1] = 0.0
    st.rhsy[1:nz + 1] = 0.0
    st.rhsz[1:nz + 1] = 0.0
    compute_dealias_convec(p, st, st.rhsx, st.rhsy, st.rhsz)
    div_stress(ops, st.rhsx, st.txx, st.txy, st.txz, True)
    div_stress(ops, st.rhsy, st.txy, st.tyy, st.tyz, True)
    bot, top = div_stress(ops, st.rhsz, st.txz, st.tyz, st.tzz, False, want_layers=True)
    st.bottom_wk_press[:] = bot
    st.top_wk_press[:] = top
    st.rhsx[1:nz + 1] = st.rhsx[1:nz + 1] + p.pfx
    st.rhsy[1:nz + 1] = st.rhsy[1:nz + 1] + p.pfy


def diagnostics(p: Params, st: State):
    """running_diagnostics.f90:148-305 -> (cfl, mke, u_star, rms_divu)."""
    nz = p.nz
    k = slice(1, nz + 1)
    umax = np.abs(st.u[k]).max()
    vmax = np.abs(st.v[k]).max()
    wmax = np.abs(st.w[k]).max()
    cfl = p.dt * (umax / p.dx + vmax / p.dy + wmax / p.dz)
    n = float(p.nx * p.ny * p.nz)
    us = st.u[k].sum() / n
    vs = st.v[k].sum() / n
    ws = (0.5 * (st.w[1:nz + 1] + st.w[2:nz + 2])).sum() / n
    mke = 0.5 * (us * us + vs * vs + ws * ws)
    ustar = st.u_star_avg.sum() / (p.nx * p.ny)
    div = st.dudx[k] + st.dvdy[k] + st.dwdz[k]
    rms = math.sqrt((div * div).sum() / n)
    return cfl, mke, ustar, rms


def les_step(ops: Ops, st: State, jt: int | None = None):
    """One pass of the LES_engine.f90:189-360 loop body."""
    p = ops.p
    nz = p.nz
    st.jt_total += 1
    jtt = st.jt_total
    jt = jtt if jt is None else jt
    if p.lbc_special == "wall_law":
        obukhov(ops, st)
        wallstress(ops, st)
    compute_vel_grad(ops, st)
    sgs_stress(ops, st, jt, jtt)
    compute_rhs_adv(ops, st)
    if jtt == 1:
        tadv1, tadv2 = 1.0, 0.0
    else:
        tadv1 = 1.5
        tadv2 = 1.0 - tadv1
    k = slice(1, nz + 1)
    st.u[k] = st.u[k] + p.dt * (tadv1 * st.rhsx[k] + tadv2 * st.rhsx_f[k])
    st.v[k] = st.v[k] + p.dt * (tadv1 * st.rhsy[k] + tadv2 * st.rhsy_f[k])
    st.w[k] = st.w[k] + p.dt * (tadv1 * st.rhsz[k] + tadv2 * st.rhsz_f[k])
    st.w[0] = 0.0
    st.w[nz + 1] = 0.0
    press_stag_array(ops, st, tadv1)
    st.u[k] = st.u[k] - p.dt * tadv1 * st.dpdx[k]
    st.v[k] = st.v[k] - p.dt * tadv1 * st.dpdy[k]
    st.w[k] = st.w[k] - p.dt * tadv1 * st.dpdz[k]
    st.rhsx[k] = st.rhsx[k] - st.dpdx[k]
    st.rhsy[k] = st.rhsy[k] - st.dpdy[k]
    st.rhsz[k] = st.rhsz[k] - st.dpdz[k]
    st.w[1] = 0.0
    st.w[nz + 1] = 0.0
    apply_bcs(p, st)
    return diagnostics(p, st)


def make_state(p: Params, seed: int = 0, amp: float = 0.1):
    st = State(p)
    u, v, w = log_law_fields(p, seed, amp)
    set_initial_conditions(p, st, u, v, w)
    return st


# ---------------------------------------------------------------------------
# checkpoint files (IO_checkpoint.f90:119-256 on a 1x1 process grid)
# ---------------------------------------------------------------------------
CHECKPOINT_FIELDS = ("u", "v", "w", "rhsx", "rhsy", "rhsz", "cs_opt2")
CHECKPOINT_F = ("F_LM", "F_MM", "F_QN", "F_NN")


def write_checkpoint(st: State, path) -> None:
    """write_checkpoint_file: each variable as nx*ny*(nz+1) native float64
    values, levels 1..nz+1 in Fortran order (write_var_tbg / write_var_tg
    start at var(1,1,1)); the F averages only when Lagran_init is set."""
    names = CHECKPOINT_FIELDS + (CHECKPOINT_F if st.lagran_init else ())
    with open(path, "wb") as f:
        for n in names:
            f.write(np.ascontiguousarray(getattr(st, n)[1:], dtype="<f8").tobytes())


def read_checkpoint(st: State, path, lagran_init: bool) -> None:
    """read_checkpoint_file + checkpoint_in: levels 1..nz+1 of each variable;
    the ghost updates of checkpoint_in do nothing on one rank.  With
    Lagran_init the Lagrangian-init flag is set (compute_LagScaleDep.f90:66)."""
    shp = st.u[1:].shape  # (nz+1, ny, nx); st.p is the pressure field
    n = int(np.prod(shp))
    names = CHECKPOINT_FIELDS + (CHECKPOINT_F if lagran_init else ())
    data = np.fromfile(path, dtype="<f8")
    if data.size < n * len(names):
        raise ValueError("[Restart error] checkpoint file too short for this grid")
    for q, name in enumerate(names):
        getattr(st, name)[1:] = data[q * n:(q + 1) * n].reshape(shp)
    for name in ("u_lag", "v_lag", "w_lag"):
        getattr(st, name)[:] = 0.0
    if lagran_init:
        st.f_coeff_init = True
        st.lagran_init = True
