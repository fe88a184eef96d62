"""FP64 CPU oracle of the scalar transport, the dynamic Prandtl model, the
buoyancy term, the sponge layer and the Coriolis forcing -- test
infrastructure only (imported by tests/, the smoke check and the bench's CPU
legs, never by the product path).

Parity unpinned: the reference's scalar module is a stub
(compute_scalars.f90:80-151 keeps only the AB2 update of step_scalars and the
ghost values theta(0) = 0, theta(nz+1) = theta(nz)), and its sponge is built
but zeroed and disconnected (sponge_damping.f90:83, LES_engine.f90:565).  The
equations here are written from the physics and from the reference's
conventions for the momentum (staggering, dealiasing, stress signs):

* theta lives on uvp nodes (compute_scalars.f90:63-65); d theta/dx, dy on uvp
  nodes (spectral, as grad_velocity_filt), d theta/dz on w nodes (ddz_uv).
  At the wall the vertical gradient is the log law of a prescribed surface
  flux q_s: d theta/dz(1) = -q_s / (kappa u* dz/2) (u* of the wall law, 0
  where u* = 0).  Ghosts: theta(0) = 0 (step_scalars), theta(nz+1) =
  theta(nz) + Gamma_top dz (the stub's rule for Gamma_top = 0).
* Convective term, rotational-form conventions of compute_convective_padd:
  -(u d_x theta + v d_y theta + (w d_z theta)(k, k+1) / 2) on uvp nodes, the
  products formed on the 3/2-padded grid (or the 2/3-truncated one).
* SGS flux with the sign of the reference's stresses (rhs += div pi):
  pi_j = nu_theta d_j theta, nu_theta = |S| (Cs^2 l^2 / Pr_t) for the
  constant-Prandtl model or |S| kappa(z) Delta^2 for the dynamic one, where
  kappa = Cs^2/Pr_t is the plane-averaged least-squares Germano coefficient
  at the 2 Delta test filter (K_j = filt(u_j theta) - filt(u_j) filt(theta),
  X_j = Delta^2 (filt(|S| d_j theta) - 4 |S~| d_j theta~), kappa =
  max(0, <K X> / <X X>)), updated at the momentum dynamic procedure's cadence
  (every cs_count steps from dyn_init; kappa = 0.03 / Pr_t before).
  pi_x, pi_y on uvp nodes (nu_theta at k and k+1 averaged, level 1 as is),
  pi_z on w nodes (k >= 2), pi_z(1) = -q_s.
* Buoyancy on w nodes k = 2..nz: rhs_z += beta (theta_w - <theta_w>),
  theta_w(k) = (theta(k) + theta(k-1)) / 2, beta = g / theta_0.
* Sponge (add_sponge_damping, sponge_damping.f90:131-161, with the profile of
  sponge_damping_init :61-80 and no zeroing): on w nodes z = (k-1) dz,
  s(k) = 3.9 (1 - cos(pi (z - z_d)/(lz - z_d))) / 2 above z_d = f lz,
  s(nz+1) = s(nz); rhs_x -= (s(k) + s(k+1))/2 (u - <u>), likewise v, and
  rhs_z -= s(k) (w - <w>), levels 1..nz.
* Coriolis (LES_engine.f90:553-561): rhs_x += f v - f v_g, rhs_y += -f u +
  f u_g, levels 1..nz.
* Scalar AB2 (step_scalars :111-135): theta += dt (tadv1 rhs + tadv2 rhs_f),
  then the ghosts.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from oracle import les_oracle as O

SCALAR_FIELDS = ("theta", "dtdx", "dtdy", "dtdz", "rhs_t", "rhs_t_f", "qx", "qy", "qz")


@dataclass
class ScalarParams:
    surface_flux: float = 0.0  # q_s, kinematic, positive upward
    top_gradient: float = 0.0  # d theta / dz at the lid
    buoyancy: float = 0.0      # g / theta_0 (0: passive scalar)
    pr_t: float = 0.4          # constant Prandtl number / initial Cs^2/Pr_t = 0.03 / pr_t
    dynamic: bool = True       # plane-averaged dynamic Cs^2 / Pr_t


@dataclass
class Forcing:
    sponge_fraction: float = 0.0  # 0: no sponge; 0.8 = top 20 %
    coriol: float = 0.0
    ug: float = 0.0
    vg: float = 0.0


def scalar_init(p: O.Params, st: O.State, sp: ScalarParams, theta=None):
    """Scalar state on an oracle State: fields zero, kappa at its initial value."""
    shp = st.u.shape
    for n in SCALAR_FIELDS:
        setattr(st, n, np.zeros(shp))
    st.kappa = np.full(p.nz + 2, 0.03 / sp.pr_t)
    st.sp = sp
    if theta is not None:
        st.theta[1:p.nz + 1] = theta
    scalar_bc(p, st)


def scalar_bc(p: O.Params, st: O.State):
    """step_scalars (compute_scalars.f90:127-133) with a lid gradient."""
    nz = p.nz
    st.theta[0] = 0.0
    st.theta[nz + 1] = st.theta[nz] + st.sp.top_gradient * p.dz


def scalar_grad(ops: O.Ops, st: O.State):
    p = ops.p
    O.grad_velocity_filt(ops, st.theta, st.dtdx, st.dtdy)
    O.ddz_uv(p, st.dtdz, st.theta)
    us = st.u_star_avg
    with np.errstate(divide="ignore", invalid="ignore"):
        g = np.where(us != 0.0, -st.sp.surface_flux / (O.KVONK * us * (0.5 * p.dz)), 0.0)
    st.dtdz[1] = g


def sgs_flux(ops: O.Ops, st: O.State, s):
    """pi_x, pi_y (uvp), pi_z (w) from the strain of compute_sij; s = the
    six S_ij arrays."""
    p = ops.p
    nz = p.nz
    k = slice(1, nz + 2)
    S = np.zeros_like(st.u)
    S[k] = O.strain_norm(*(x[k] for x in s))
    sp = st.sp
    if sp.dynamic:
        nut = S * (st.kappa * ops.delta ** 2)[:, None, None]
    else:
        # the momentum model's nu_t (Cs^2 l^2 |S|, mixing length of sgs_stress) over Pr_t
        nut = st.nu_t / sp.pr_t
    st.qx[1] = nut[1] * st.dtdx[1]
    st.qy[1] = nut[1] * st.dtdy[1]
    kk = slice(2, nz + 1)
    kp = slice(3, nz + 2)
    c = 0.5 * (nut[kk] + nut[kp])
    st.qx[kk] = c * st.dtdx[kk]
    st.qy[kk] = c * st.dtdy[kk]
    k2 = slice(2, nz + 2)
    st.qz[k2] = nut[k2] * st.dtdz[k2]
    st.qz[1] = -sp.surface_flux


def dynamic_kappa(ops: O.Ops, st: O.State, s):
    """Plane-averaged Germano coefficient Cs^2/Pr_t at the 2 Delta filter on
    levels 1..nz+1, the node conventions of compute_dynamic_mum
    (compute_LagScaleDep.f90:501-584: level 1 on uvp nodes, u, v, w there
    as u(1), v(1), w(2)/4; levels >= 2 on w nodes)."""
    p = ops.p
    nz = p.nz
    shp = st.u.shape
    k = slice(2, nz + 2)
    km = slice(1, nz + 1)

    def to_w(f, first):
        g = np.zeros(shp)
        g[1] = first
        g[k] = 0.5 * (f[k] + f[km])
        return g

    uf = to_w(st.u, st.u[1])
    vf = to_w(st.v, st.v[1])
    wf = np.zeros(shp)
    wf[1] = 0.25 * st.w[2]
    wf[k] = st.w[k]
    tf = to_w(st.theta, st.theta[1])
    tx = to_w(st.dtdx, st.dtdx[1])
    ty = to_w(st.dtdy, st.dtdy[1])
    tz = st.dtdz.copy()
    S = np.zeros(shp)
    S[1:] = O.strain_norm(*(x[1:] for x in s))
    prods = [uf * tf, vf * tf, wf * tf]
    st_s = [S * tx, S * ty, S * tz]
    filt = [x.copy() for x in [uf, vf, wf, tf] + prods + list(s) + [tx, ty, tz] + st_s]
    for f in filt:
        O.test_filter(ops, f, ops.g_test)
    uF, vF, wF, tF = filt[0:4]
    utF, vtF, wtF = filt[4:7]
    sF = filt[7:13]
    txF, tyF, tzF = filt[13:16]
    stx, sty, stz = filt[16:19]
    s_ft = O.strain_norm(*sF)
    d2 = ops.delta ** 2
    K = [utF - uF * tF, vtF - vF * tF, wtF - wF * tF]
    X = [d2 * (stx - 4.0 * s_ft * txF), d2 * (sty - 4.0 * s_ft * tyF), d2 * (stz - 4.0 * s_ft * tzF)]
    kx = K[0] * X[0] + K[1] * X[1] + K[2] * X[2]
    xx = X[0] * X[0] + X[1] * X[1] + X[2] * X[2]
    kk = slice(1, nz + 2)
    num = kx[kk].sum(axis=(1, 2)) / (p.nx * p.ny)
    den = xx[kk].sum(axis=(1, 2)) / (p.nx * p.ny)
    c = np.where(den != 0.0, num / np.where(den != 0.0, den, 1.0), 0.0)
    st.kappa[1:nz + 2] = np.maximum(0.0, c)


def scalar_sgs(ops: O.Ops, st: O.State, jt: int, jtt: int):
    """After sgs_stress of the same step (nu_t formed): kappa update at the
    dynamic cadence, then the fluxes."""
    p = ops.p
    s = O.compute_sij(p, st)
    if st.sp.dynamic and jtt >= p.dyn_init and jt % p.cs_count == 0:
        dynamic_kappa(ops, st, s)
    sgs_flux(ops, st, s)


def scalar_convec(p: O.Params, st: O.State):
    """-(u . grad theta) on uvp levels 1..nz with the momentum's dealiasing."""
    nz = p.nz
    const = 1.0 / (p.nx * p.ny)
    to_big = O.transpose_to_big if p.dealias == "padd" else O.transpose_to_truncate
    ub = to_big(p, -const * st.u)
    vb = to_big(p, -const * st.v)
    wb = to_big(p, -const * st.w)
    tx = to_big(p, const * st.dtdx)
    ty = to_big(p, const * st.dtdy)
    tz = to_big(p, const * st.dtdz)
    if p.dealias == "padd":
        c = 1.0 / ((3 * p.nx // 2) * (3 * p.ny // 2))
        back = O.dealias_padd
    else:
        c = 1.0 / (p.nx * p.ny)
        back = O.dealias_trunc
    k = slice(1, nz + 1)
    kp = slice(2, nz + 2)
    wk = c * (ub[k] * tx[k] + vb[k] * ty[k] + 0.5 * (wb[k] * tz[k] + wb[kp] * tz[kp]))
    out = np.zeros_like(st.u)
    out[k] = back(p, wk)
    return out


def plane_mean(f):
    return f.sum(axis=(-2, -1)) / (f.shape[-1] * f.shape[-2])


def sponge_profile(p: O.Params, frac: float):
    """sponge_damping.f90:61-80 (w nodes, z = (k-1) dz, k = 1..nz+1)."""
    s = np.zeros(p.nz + 2)
    if frac <= 0.0:
        return s
    z_d = frac * p.lz
    for k in range(1, p.nz + 2):
        z = (1 + k - 2.0) * p.dz
        if z_d <= z <= p.lz:
            s[k] = 3.9 * 0.5 * (1.0 - math.cos(O.PI * (z - z_d) / (p.lz - z_d)))
    s[p.nz + 1] = s[p.nz]
    return s


def forcing(p: O.Params, st: O.State, fc: Forcing):
    """Coriolis (LES_engine.f90:553-561) then the sponge (sponge_damping.f90:131-161)."""
    nz = p.nz
    k = slice(1, nz + 1)
    if fc.coriol != 0.0:
        u, v = st.u[k].copy(), st.v[k].copy()
        st.rhsx[k] = st.rhsx[k] + fc.coriol * v - fc.coriol * fc.vg
        st.rhsy[k] = st.rhsy[k] - fc.coriol * u + fc.coriol * fc.ug
    if fc.sponge_fraction > 0.0:
        s = sponge_profile(p, fc.sponge_fraction)
        ua = plane_mean(st.u[k])
        va = plane_mean(st.v[k])
        wa = plane_mean(st.w[k])
        sh = (0.5 * (s[1:nz + 1] + s[2:nz + 2]))[:, None, None]
        st.rhsx[k] = st.rhsx[k] - sh * (st.u[k] - ua[:, None, None])
        st.rhsy[k] = st.rhsy[k] - sh * (st.v[k] - va[:, None, None])
        st.rhsz[k] = st.rhsz[k] - s[1:nz + 1, None, None] * (st.w[k] - wa[:, None, None])


def buoyancy(p: O.Params, st: O.State):
    nz = p.nz
    beta = st.sp.buoyancy
    if beta == 0.0:
        return
    tm = plane_mean(st.theta)
    k = slice(2, nz + 1)
    km = slice(1, nz)
    tw = 0.5 * (st.theta[k] + st.theta[km])
    twm = 0.5 * (tm[k] + tm[km])
    st.rhsz[k] = st.rhsz[k] + beta * (tw - twm[:, None, None])


def scalar_rhs(ops: O.Ops, st: O.State):
    p = ops.p
    nz = p.nz
    st.rhs_t_f[1:nz + 1] = st.rhs_t[1:nz + 1]
    conv = scalar_convec(p, st)
    st.rhs_t[1:nz + 1] = conv[1:nz + 1]
    O.div_stress(ops, st.rhs_t, st.qx, st.qy, st.qz, True)


def les_step(ops: O.Ops, st: O.State, fc: Forcing | None = None, jt: int | None = None):
    """One time step of the momentum (les_oracle.les_step) with the scalar,
    buoyancy and forcing terms inserted where they act."""
    p = ops.p
    nz = p.nz
    fc = fc or Forcing()
    has_t = hasattr(st, "theta")
    st.jt_total += 1
    jtt = st.jt_total
    jt = jtt if jt is None else jt
    if p.lbc_special == "wall_law":
        O.obukhov(ops, st)
        O.wallstress(ops, st)
    O.compute_vel_grad(ops, st)
    if has_t:
        scalar_grad(ops, st)
    O.sgs_stress(ops, st, jt, jtt)
    if has_t:
        scalar_sgs(ops, st, jt, jtt)
    O.compute_rhs_adv(ops, st)
    forcing(p, st, fc)
    if has_t:
        scalar_rhs(ops, st)
        buoyancy(p, st)
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
    if has_t:
        st.theta[k] = st.theta[k] + p.dt * (tadv1 * st.rhs_t[k] + tadv2 * st.rhs_t_f[k])
        scalar_bc(p, st)
    O.press_stag_array(ops, st, tadv1)
    st.u[k] = st.u[k] - p.dt * tadv1 * st.dpdx[k]
    st.v[k] = st.v[k] - p.dt * tadv1 * st.dpdy[k]
    st.w[k] = st.w[k] - p.dt * tadv1 * st.dpdz[k]
    st.rhsx[k] = st.rhsx[k] - st.dpdx[k]
    st.rhsy[k] = st.rhsy[k] - st.dpdy[k]
    st.rhsz[k] = st.rhsz[k] - st.dpdz[k]
    st.w[1] = 0.0
    st.w[nz + 1] = 0.0
    O.apply_bcs(p, st)
    return O.diagnostics(p, st)


def linear_profile(p: O.Params, seed: int = 0, amp: float = 0.01, gradient: float = 1.0):
    """Config-2 passive scalar: theta = gradient * z at the uvp heights plus
    seeded uniform noise of +-amp (the velocity's counter-based generator,
    stream 3)."""
    z = (np.arange(1, p.nz + 1) - 0.5) * p.dz
    th = gradient * z[:, None, None] + np.zeros((p.nz, p.ny, p.nx))
    return th + amp * O.rng_uniform(seed, 3, th.shape)


def inversion_profile(p: O.Params, seed: int = 0, z_inv: float = 0.5, lapse: float = 10.0, amp: float = 0.1,
                      z_noise: float = 0.1):
    """Convective-boundary-layer temperature (departure from theta_0): 0 up to
    z_inv, lapse * (z - z_inv) above (0.01 K/m with z_i = 1000 m is 10 K per
    unit height), +-amp K seeded noise below z_noise."""
    z = (np.arange(1, p.nz + 1) - 0.5) * p.dz
    base = np.where(z > z_inv, lapse * (z - z_inv), 0.0)
    th = base[:, None, None] + np.zeros((p.nz, p.ny, p.nx))
    noise = amp * O.rng_uniform(seed, 3, th.shape)
    return th + np.where((z < z_noise)[:, None, None], noise, 0.0)
