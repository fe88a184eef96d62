"""Shared helpers for the parity tests: mirror an oracle state into the GPU
library and compare the two states field by field."""
from __future__ import annotations

import numpy as np

from oracle import les_oracle as O

PLANE_NAMES = ("lbc_u", "lbc_v", "lbc_w", "ubc_u", "ubc_v", "ubc_w", "bottom_wk_press", "top_wk_press",
               "lbc_z0", "u_star_avg")
BC_CODE = {"drc": 1, "neu": 2}


def oracle_params(**kw) -> O.Params:
    return O.Params(**kw)


def run_params(op: O.Params):
    """RunParams of the library with the same namelist values as an oracle Params."""
    from new_repo_b200 import RunParams

    return RunParams(nx=op.nx, ny=op.ny, nz=op.nz, dt=op.dt, xy_pi=op.xy_pi, lx_in=op.lx_in, ly_in=op.ly_in,
                     lz_in=op.lz_in, zi=op.zi, u_scale=op.u_scale, lbc_dz0=op.lbc_dz0, pfx=op.pfx, pfy=op.pfy,
                     cs0=op.cs0, sgs_model=op.sgs_model, cs_count=op.cs_count, dyn_init=op.dyn_init,
                     lbc_special=op.lbc_special, wall_model=op.wall_model, dealias=op.dealias,
                     lag_halo=op.lag_halo)


def oracle_run(p: O.Params, nsteps: int, seed: int = 0):
    ops = O.Ops(p)
    st = O.make_state(p, seed=seed)
    for _ in range(nsteps):
        O.les_step(ops, st)
    return ops, st


def mirror(les, st: O.State):
    """Upload every field, plane and flag of an oracle state."""
    for n in O.FIELDS:
        les.upload(n, getattr(st, n))
    for n in PLANE_NAMES:
        les.upload_plane(n, getattr(st, n))
    les.set_bc_types([BC_CODE.get(st.lbc_typ[c], 0) for c in "uvw"], [BC_CODE.get(st.ubc_typ[c], 0) for c in "uvw"])
    les.f_coeff_init = st.f_coeff_init
    les.jt_total = st.jt_total
    les.jt = st.jt_total


def rel_err(a, b) -> float:
    """Normwise relative error max|a - b| / max|b| over the entries that are
    not the reference's BOGUS sentinel; sentinel entries must match to 1e-6."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    m = b == O.BOGUS
    if m.any() and not np.allclose(a[m], b[m], rtol=1e-6, atol=0):
        return 1.0
    a, b = a[~m], b[~m]
    if b.size == 0:
        return 0.0
    den = np.abs(b).max()
    num = np.abs(a - b).max()
    if den == 0.0:
        return float(num)
    return float(num / den)


def field_errors(les, st: O.State, names=None):
    """rel_err per field and plane between the GPU state and the oracle state."""
    names = O.FIELDS if names is None else names
    out = {}
    for n in names:
        out[n] = rel_err(les.download(n), getattr(st, n))
    for n in PLANE_NAMES:
        out[n] = rel_err(les.download_plane(n), getattr(st, n))
    return out


def worst(errs: dict):
    k = max(errs, key=errs.get)
    return k, errs[k]


def rel_err_real4(a, b, tol: float, ulp_rel: float = 2.5e-7, max_frac: float = 1e-5):
    """rel_err for fields that pass through the reference's REAL(4) roundings
    (compute_LagScaleDep.f90:624-690 rounds cs_opt2, beta, F_LM and F_QN to
    single precision).  Two FP64 computations that differ by one FP64 ulp
    can round a value to neighbouring floats, which moves that point (and
    nu_t, tau there) by about one float ulp.  Points above the FP64 bar are
    accepted when they differ by 2e-8 .. `ulp_rel` of their own value and
    are rare (at most max(4, max_frac of the points)); returns the normwise
    error over the remaining points and the number of such points."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    m = b == O.BOGUS
    if m.any() and not np.allclose(a[m], b[m], rtol=1e-6, atol=0):
        return 1.0, 0
    a, b = a[~m], b[~m]
    if b.size == 0:
        return 0.0, 0
    den = np.abs(b).max()
    d = np.abs(a - b)
    over = d > tol * den
    flips = over & (d <= ulp_rel * np.abs(b)) & (d >= 2e-8 * np.abs(b))  # one float ulp is 6e-8 .. 1.2e-7
    if flips.sum() > max(4, int(max_frac * b.size)):
        return float(d.max() / den), int(flips.sum())
    rest = d[~flips]
    return (float(rest.max() / den) if rest.size else 0.0), int(flips.sum())
