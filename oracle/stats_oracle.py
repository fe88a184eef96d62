"""CPU FP64 oracle for the post-step statistics -- TEST INFRASTRUCTURE ONLY.

Restates, on one rank, the running sums of ``src/IO_statistics.f90`` and the
plane-averaged TKE budget of ``src/tke_budget1D.f90``.  Only ``tests/`` may
import it, as the checker for ``les_stat_*`` / ``les_tke_*``.

Parity status: unpinned (the reference ships no statistics fixtures and
cannot be built here); the restatement follows the Fortran statement by
statement, with these behaviours of the source kept:

* ``Mav_uw`` / ``Mav_vw`` level 1 is reset to zero on every call
  (IO_statistics.f90:378-384).
* The budget's ``cs`` profile reads ``cs_opt2`` one level up: ``scr1 =
  cs_opt2`` copies an ``(nx,ny,nz+1)`` array into an ``(nx,ny,0:nz+1)``
  scratch by array position (tke_budget1D.f90:275), so scratch level k holds
  cs_opt2 level k+1.  The same copy leaves cs_opt2 level 1 in scratch level 0,
  which is still there when the cleaned pressure is built in that scratch
  (:336-343) and reaches the ``dpdz`` profile at level 1 through ddz_uv.
  Scratch level nz+1 is never set by the routine; it is taken as zero
  (it reaches only ``dpdz`` at level nz).
* Budget records are ``avar / tke_period`` whatever the number of steps
  summed, written at ``mod(jt, tke_period) == 0`` (jt, not jt_total).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from .les_oracle import Ops, State, grad_velocity_filt, ddz_uv

# IO_statistics.f90:447-488, the order of the RAV_*_3D.dat records
STAT_NAMES = ("u", "v", "w", "p", "u2", "v2", "w2", "u3", "v3", "w3", "u4", "v4", "w4", "uv", "uw", "vw",
              "txx", "tyy", "tzz", "txy", "txz", "tyz", "dudz", "dvdz", "nut", "cs")

# tke_budget1D.f90:218-383, the order of the avg_var calls
TKE_NAMES = ("u", "v", "w", "dudx", "dudy", "dudz", "dvdx", "dvdy", "dvdz", "dwdx", "dwdy", "dwdz",
             "uu", "vv", "ww", "uv", "uw", "vw", "txx", "tyy", "tzz", "txy", "txz", "tyz", "cs",
             "uuw", "vvw", "www", "uww", "wtzz", "utxz", "vtyz", "dxx", "dyy", "dzz", "dxy", "dxz", "dyz",
             "dudx2", "dudy2", "dudz2", "dvdx2", "dvdy2", "dvdz2", "dwdx2", "dwdy2", "dwdz2",
             "dudxdwdx", "dudydwdy", "dudzdwdz",
             "p", "dpdx", "dpdy", "dpdz", "pw", "pu", "pdudx", "pdvdy", "pdwdz", "pdwdx", "pdudz")

SPECTRA_WINDOWS = (1500000, 1550000, 1600000, 1650000)  # IO_statistics.f90:566-581


class RunningStats:
    """Module state of IO_statistics.f90 (io_stat_init :40-250)."""

    def __init__(self, p):
        self.p = p
        self.sums = np.zeros((len(STAT_NAMES), p.nz, p.ny, p.nx))
        self.ustar = np.zeros((p.ny, p.nx))
        self.iterations = 0


def stat_averages(rs: RunningStats, st: State, jt: int, jt_total: int, start_stats: int, running_period: int,
                  out_path: str | None = None) -> bool:
    """io_stat_averages (IO_statistics.f90:265-291) with io_2D_stat_averages
    (:300-354) and io_3D_stat_averages (:363-518).  Returns True when the
    sums were written (and restarted)."""
    p = rs.p
    nz = p.nz
    rs.iterations += 1
    write = (jt_total % running_period == 0) and jt_total > start_stats
    base = None if out_path is None else f"{out_path}RAV_{jt_total:09d}"
    if write:
        if base is not None:
            Path(base + "_info.txt").write_text(f"{p.nx:6d}{p.ny:6d}{p.nz:6d}{rs.iterations:10d}\n")
        rs.iterations = 0
    rs.ustar += st.u_star_avg
    if write:
        if base is not None:
            rs.ustar.astype("<f8").tofile(base + "_2D.dat")
        rs.ustar[:] = 0.0
    k = slice(1, nz + 1)
    u, v, w = st.u[k], st.v[k], st.w[k]
    u2, v2, w2 = u * u, v * v, w * w
    s = rs.sums
    s[0] += u
    s[1] += v
    s[2] += w
    s[3] += st.p[k]
    s[4] += u2
    s[5] += v2
    s[6] += w2
    s[7] += u2 * u
    s[8] += v2 * v
    s[9] += w2 * w
    s[10] += u2 * u2
    s[11] += v2 * v2
    s[12] += w2 * w2
    s[13] += u * v
    s[14][0] = 0.0
    s[15][0] = 0.0
    s[14][1:] += st.w[2:nz + 1] * (0.5 * (st.u[1:nz] + st.u[2:nz + 1]))
    s[15][1:] += st.w[2:nz + 1] * (0.5 * (st.v[1:nz] + st.v[2:nz + 1]))
    for q, n in enumerate(("txx", "tyy", "tzz", "txy", "txz", "tyz", "dudz", "dvdz", "nu_t")):
        s[16 + q] += getattr(st, n)[k]
    s[25] += np.sqrt(st.cs_opt2[k])
    if write:
        if base is not None:
            s.astype("<f8").tofile(base + "_3D.dat")
        s[:] = 0.0
    return write


def spectra_due(jt: int, jt_total: int) -> bool:
    """io_stat_spectra's windows (IO_statistics.f90:566-581)."""
    return any(lo <= jt_total <= lo + 2000 and jt % 10 == 0 for lo in SPECTRA_WINDOWS)


def _int(f):
    """int_var (tke_budget1D.f90:424-446): w node -> uvp node, levels 1..nz."""
    return 0.5 * (f[1:-1] + f[2:])


def tke_pointwise(ops: Ops, st: State, wall_law: bool):
    """The 61 pointwise quantities of compute_tke_budget (tke_budget1D.f90:
    209-390) on levels 1..nz, as a dict name -> (nz, ny, nx)."""
    p = ops.p
    nz = p.nz
    k = slice(1, nz + 1)
    q = {}
    U, V = st.u[k], st.v[k]
    W = _int(st.w)
    ux, uy, uz = st.dudx[k], st.dudy[k], _int(st.dudz)
    vx, vy, vz = st.dvdx[k], st.dvdy[k], _int(st.dvdz)
    wx, wy, wz = _int(st.dwdx), _int(st.dwdy), st.dwdz[k]
    for n, a in (("u", U), ("v", V), ("w", W), ("dudx", ux), ("dudy", uy), ("dudz", uz), ("dvdx", vx),
                 ("dvdy", vy), ("dvdz", vz), ("dwdx", wx), ("dwdy", wy), ("dwdz", wz)):
        q[n] = a
    q["uu"], q["vv"], q["ww"] = U * U, V * V, W * W
    q["uv"], q["uw"], q["vw"] = U * V, W * U, W * V
    txx, tyy, tzz, txy = st.txx[k], st.tyy[k], st.tzz[k], st.txy[k]
    txzi, tyzi = _int(st.txz), _int(st.tyz)
    q["txx"], q["tyy"], q["tzz"], q["txy"], q["txz"], q["tyz"] = txx, tyy, tzz, txy, txzi, tyzi
    q["cs"] = st.cs_opt2[2:nz + 2]  # scratch level k = cs_opt2 level k+1 (array copy by position)
    q["uuw"] = (U * U) * W
    q["vvw"] = (V * V) * W
    q["www"] = (W * W) * W
    q["uww"] = U * (W * W)
    q["wtzz"] = W * tzz
    s3, s2 = txzi.copy(), tyzi.copy()
    s4 = _int(st.dudz + st.dwdx)
    s1 = _int(st.dvdz + st.dwdy)
    if wall_law:
        s3[0] = st.txz[1]
        s2[0] = st.tyz[1]
        s4[0] = st.dudz[1] + 0.5 * (st.dwdx[1] + st.dwdx[2])
        s1[0] = st.dvdz[1] + 0.5 * (st.dwdy[1] + st.dwdy[2])
    q["utxz"], q["vtyz"] = s3 * U, s2 * V
    q["dxx"], q["dyy"], q["dzz"] = ux * txx, vy * tyy, wz * tzz
    q["dxy"] = 0.5 * (uy + vx) * txy
    q["dxz"] = 0.5 * s4 * s3
    q["dyz"] = 0.5 * s2 * s1
    for n, a in (("dudx2", ux), ("dudy2", uy), ("dudz2", uz), ("dvdx2", vx), ("dvdy2", vy), ("dvdz2", vz),
                 ("dwdx2", wx), ("dwdy2", wy), ("dwdz2", wz)):
        q[n] = a * a
    q["dudxdwdx"], q["dudydwdy"], q["dudzdwdz"] = ux * wx, uy * wy, uz * wz
    # pressure terms (:336-372) on a (0:nz+1) scratch
    c = np.zeros_like(st.p)
    c[1:nz + 1] = st.p[k] - 0.5 * (U ** 2 + V ** 2 + (0.5 * (st.w[1:nz + 1] + st.w[2:nz + 2])) ** 2)
    c[0] = st.cs_opt2[1]
    c[nz + 1] = 0.0
    cx, cy = np.zeros_like(c), np.zeros_like(c)
    grad_velocity_filt(ops, c, cx, cy)  # c becomes its Nyquist-filtered self
    dcdz = np.zeros_like(c)
    ddz_uv(p, dcdz, c)
    C = c[k]
    q["p"], q["dpdx"], q["dpdy"] = C, cx[k], cy[k]
    q["dpdz"] = _int(dcdz)
    q["pw"], q["pu"] = C * W, C * U
    q["pdudx"], q["pdvdy"], q["pdwdz"] = C * ux, C * vy, C * wz
    q["pdwdx"], q["pdudz"] = C * wx, C * uz
    assert len(q) == len(TKE_NAMES) and set(q) == set(TKE_NAMES)
    return q


def tke_profiles(ops: Ops, st: State, wall_law: bool):
    """(61, nz) plane averages (compute_planar_average, utility_tools.f90:
    59-92) and a per-quantity scale (max over levels of the mean |value|)."""
    p = ops.p
    q = tke_pointwise(ops, st, wall_law)
    means = np.stack([q[n].sum(axis=(1, 2)) / (p.nx * p.ny) for n in TKE_NAMES])
    scale = np.array([np.abs(q[n]).mean(axis=(1, 2)).max() for n in TKE_NAMES])
    return means, scale


class TkeBudget:
    """Module state of tke_budget1D.f90 (tke_budget_init :61-160)."""

    def __init__(self, p, out_path: str | None = None):
        self.p = p
        self.avar = np.zeros((len(TKE_NAMES), p.nz))
        self.ii = 1
        self.dir = None if out_path is None else Path(f"{out_path}ta1_profiles")
        if self.dir is not None:
            self.dir.mkdir(exist_ok=True)


def compute_tke_budget(tb: TkeBudget, ops: Ops, st: State, jt: int, tke_period: int, wall_law: bool) -> bool:
    """compute_tke_budget(jt) (tke_budget1D.f90:209-390) with avg_var
    (:396-420).  Returns True when a record was written."""
    means, _ = tke_profiles(ops, st, wall_law)
    tb.avar += means
    if jt % tke_period != 0:
        return False
    if tb.dir is not None:
        nz = tb.p.nz
        for qi, n in enumerate(TKE_NAMES):
            path = tb.dir / f"{n}.out"
            mode = "r+b" if path.exists() else "w+b"
            with open(path, mode) as f:
                f.seek((tb.ii - 1) * 8 * nz)
                f.write((tb.avar[qi] / float(tke_period)).astype("<f8").tobytes())
    tb.avar[:] = 0.0
    tb.ii += 1
    return True
