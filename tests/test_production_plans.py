"""Parity of the SGS, wall-law, stress-divergence and pressure operators at
production plan lengths, against the FP64 oracle.

The per-operator tests of the full step run on 32- and 64-point grids; the
bench runs 256-point plans (and 512 for the large case), where the LASD test
filters keep only nk2 / nk4 spectral columns, the 21-field combining pass
runs on 256- or 512-point x rows, and the wall layer filters one level.  Here
those paths run on a few levels of nx = ny = 256 and 512 grids.  The
tridiagonal solve is checked on a tall column grid (L = 258 levels).

Tolerances (normwise relative per field, BOGUS entries excluded): FP64
<= 1e-12; mixed precision <= 1e-5 on FP32-rounded inputs.
"""
import numpy as np
import pytest

from oracle import les_oracle as O
from tests.helpers import mirror, rel_err, rel_err_real4, run_params

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "mixed": 1e-5}
SGS_NAMES = ("cs_opt2", "nu_t", "txx", "txy", "txz", "tyy", "tyz", "tzz", "F_LM", "F_MM", "F_QN", "F_NN", "beta")


def _round_f32(st):
    for n in O.FIELDS + O.PLANES:
        a = getattr(st, n)
        a[...] = a.astype(np.float32).astype(np.float64)


def _les(p, precision):
    from new_repo_b200 import LES

    return LES(run_params(p), precision=precision)


def _lasd_state(n, jtt, seed=3, nz=4):
    """A state just before a LASD update at step jtt (cs_count 5, dyn_init 5):
    gradients of a log-law + noise field, Lagrangian accumulators holding
    four steps of u, and (jtt = 10) positive Lagrangian averages F_* from a
    previous update."""
    p = O.Params(nx=n, ny=n, nz=nz, dt=1e-4, sgs_model="dyn_LagScaleDep")
    ops = O.Ops(p)
    st = O.make_state(p, seed=seed)
    O.obukhov(ops, st)
    O.wallstress(ops, st)
    O.compute_vel_grad(ops, st)
    for f in ("u", "v", "w"):
        lag = getattr(st, f + "_lag")
        lag[1:] = 4.0 * getattr(st, f)[1:]
        lag[0] = 0.0
    if jtt > 5:
        rng = np.random.default_rng(seed)
        shp = st.F_MM[1:].shape
        st.F_MM[1:] = 1e-3 * (1.0 + 0.5 * rng.random(shp))
        st.F_LM[1:] = 0.03 * st.F_MM[1:] * (1.0 + 0.2 * rng.random(shp))
        st.F_NN[1:] = 2e-3 * (1.0 + 0.5 * rng.random(shp))
        st.F_QN[1:] = 0.03 * st.F_NN[1:] * (1.0 + 0.2 * rng.random(shp))
        st.f_coeff_init = True
        st.lagran_init = True
    return p, ops, st


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("jtt", [5, 10])
@pytest.mark.parametrize("n", [256, 512])
def test_sgs_lasd_update_large(gpu, n, jtt, precision):
    """compute_LagScaleDep_coeff at an update step: jtt = 5 initialises the
    Lagrangian averages, jtt = 10 interpolates them along the accumulated
    trajectories (k_lag_interp) before the relaxation (k_lasd_update); both
    run the 2-Delta and 4-Delta test filters of the 21 products (XF_LASD,
    YP_FILTER2, XI_LASD on nk2 / nk4 columns)."""
    p, ops, st = _lasd_state(n, jtt)
    if precision == "mixed":
        _round_f32(st)
    les = _les(p, precision)
    mirror(les, st)
    O.sgs_stress(ops, st, jtt, jtt)
    les.sgs_stress(jtt, jtt)
    for name in SGS_NAMES:
        # FP64: a REAL(4) rounding of the reference may land on the other
        # float at a few points (rel_err_real4); mixed precision: the 1e-5
        # bar covers a float ulp
        e, nflip = rel_err_real4(les.download(name)[1:], getattr(st, name)[1:], TOL[precision])
        assert e <= TOL[precision], (n, jtt, precision, name, e, nflip)
    les.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("model", ["wall_filter", "wall_inst", "wall_homog"])
@pytest.mark.parametrize("n", [256, 512])
def test_wall_law_large(gpu, n, model, precision):
    """obukhov + wallstress: the 2-Delta filtered first level (XI_WALL on nk2
    columns for wall_filter), u*, the lower boundary values, txz/tyz and
    dudz/dvdz at level 1."""
    p = O.Params(nx=n, ny=n, nz=4, dt=1e-4, wall_model=model)
    ops = O.Ops(p)
    st = O.make_state(p, seed=6)
    O.compute_vel_grad(ops, st)
    if precision == "mixed":
        _round_f32(st)
    les = _les(p, precision)
    mirror(les, st)
    O.obukhov(ops, st)
    O.wallstress(ops, st)
    les.obukhov()
    les.wallstress()
    for name in ("txz", "tyz", "dudz", "dvdz"):
        e = rel_err(les.download(name)[1], getattr(st, name)[1])
        assert e <= TOL[precision], (n, model, precision, name, e)
    for name in ("u_star_avg", "lbc_u", "lbc_v"):
        e = rel_err(les.download_plane(name), getattr(st, name))
        assert e <= TOL[precision], (n, model, precision, name, e)
    les.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("stag", [True, False])
@pytest.mark.parametrize("n", [256, 512])
def test_div_stress_large(gpu, n, stag, precision):
    """div_stress on stresses of a constant-Smagorinsky state, for both
    staggerings; stag = False also writes bottom_wk_press / top_wk_press."""
    p = O.Params(nx=n, ny=n, nz=4, dt=1e-4, sgs_model="cst_Smag")
    ops = O.Ops(p)
    st = O.make_state(p, seed=7)
    O.obukhov(ops, st)
    O.wallstress(ops, st)
    O.compute_vel_grad(ops, st)
    O.sgs_stress(ops, st, 1, 1)
    rng = np.random.default_rng(7)
    for r in ("rhsx", "rhsz"):
        getattr(st, r)[...] = rng.standard_normal(st.u.shape)
    if precision == "mixed":
        _round_f32(st)
    les = _les(p, precision)
    mirror(les, st)
    if stag:
        O.div_stress(ops, st.rhsx, st.txx, st.txy, st.txz, True)
        les.div_stress("rhsx", "txx", "txy", "txz", True)
        checks = [("rhsx", les.download("rhsx")[1:-1], st.rhsx[1:-1])]
    else:
        bot, top = O.div_stress(ops, st.rhsz, st.txz, st.tyz, st.tzz, False, want_layers=True)
        les.div_stress("rhsz", "txz", "tyz", "tzz", False)
        checks = [("rhsz", les.download("rhsz")[1:-1], st.rhsz[1:-1]),
                  ("bottom_wk_press", les.download_plane("bottom_wk_press"), bot),
                  ("top_wk_press", les.download_plane("top_wk_press"), top)]
    for name, a, b in checks:
        e = rel_err(a, b)
        assert e <= TOL[precision], (n, stag, precision, name, e)
    les.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tridiagonal_tall_column(gpu, precision):
    """press_stag_array on a 16 x 16 x 256 grid: 258 unknowns per (kx, ky)
    system (the 256^3 solve's length), against the oracle's Thomas sweep."""
    p = O.Params(nx=16, ny=16, nz=256, dt=1e-4, sgs_model="cst_Smag")
    ops = O.Ops(p)
    st = O.make_state(p, seed=8)
    rng = np.random.default_rng(8)
    for f in ("u", "v", "w"):
        getattr(st, f)[1:-1] += 0.05 * rng.standard_normal(st.u[1:-1].shape)
    st.w[0] = 0.0
    st.w[-1] = 0.0
    st.bottom_wk_press[:] = rng.standard_normal(st.bottom_wk_press.shape)
    st.top_wk_press[:] = rng.standard_normal(st.top_wk_press.shape)
    if precision == "mixed":
        _round_f32(st)
    les = _les(p, precision)
    mirror(les, st)
    O.press_stag_array(ops, st, 1.5)
    les.press_stag_array(1.5)
    for name in ("p", "dpdx", "dpdy", "dpdz"):
        a, b = les.download(name), getattr(st, name)
        if name == "p":
            a, b = a[:-1], b[:-1]
        e = rel_err(a, b)
        assert e <= TOL[precision], (precision, name, e)
    assert les.status() == 0
    les.close()


# Stated per-field bars of a 10-step mixed-precision run against the FP64
# oracle from the same FP64 initial fields (LASD updates at steps 5 and 10),
# each normwise relative to that field's own largest value.  Measured on a
# B200 (32^3 / 64x32x16): u 5e-7, v 1.4e-5, w 3.3e-5 (v and w are the +-0.1
# noise, so relative to the mean flow their error is ~1e-7); gradients and
# pressure gradients up to 1.0e-4; SGS coefficient, stresses and rhs up to
# 1.6e-4.  The FP32 storage rounding of every step and the FP32 dynamic
# procedure (ratios of small test-filtered contractions) set these levels;
# the bars leave a factor ~3.
HORIZON_TOL = {"velocity": 1e-4, "resolved": 3e-4, "sgs": 1e-3}
VEL = ("u", "v", "w")
RESOLVED = ("dudx", "dudy", "dudz", "dvdx", "dvdy", "dvdz", "dwdx", "dwdy", "dwdz", "p", "dpdx", "dpdy", "dpdz")
SGS = ("cs_opt2", "nu_t", "txx", "txy", "txz", "tyy", "tyz", "tzz", "rhsx", "rhsy", "rhsz")


@pytest.mark.parametrize("grid", [dict(nx=32, ny=32, nz=32), dict(nx=64, ny=32, nz=16)])
def test_mixed_ten_step_horizon(gpu, grid):
    p = O.Params(**grid)
    ops = O.Ops(p)
    st = O.make_state(p, seed=0)
    les = _les(p, "mixed")
    les.set_initial_conditions(*O.log_law_fields(p, seed=0))
    for _ in range(10):
        O.les_step(ops, st)
        les.step()
    errs = {}
    for group, names in (("velocity", VEL), ("resolved", RESOLVED), ("sgs", SGS)):
        for n in names:
            a, b = les.download(n), getattr(st, n)
            if n == "p":
                a, b = a[:-1], b[:-1]
            errs[n] = (group, rel_err(a[1:], b[1:]))
    report = ", ".join(f"{n}={e:.1e}" for n, (_, e) in errs.items())
    print("mixed 10-step errors:", report)
    for n, (group, e) in errs.items():
        assert e <= HORIZON_TOL[group], f"{n}: {e:.2e} > {HORIZON_TOL[group]:.0e} ({report})"
    assert les.status() == 0
    les.close()


def _advance(p, seed=9, tadv1=1.5):
    """An oracle state just before press_stag_array: the part of
    LES_engine.f90:189-283 that precedes it, on a state with a previous rhs."""
    ops = O.Ops(p)
    st = O.make_state(p, seed=seed)
    for _ in range(2):
        O.les_step(ops, st)
    st.jt_total += 1
    O.obukhov(ops, st)
    O.wallstress(ops, st)
    O.compute_vel_grad(ops, st)
    O.sgs_stress(ops, st, st.jt_total, st.jt_total)
    O.compute_rhs_adv(ops, st)
    k = slice(1, p.nz + 1)
    for f, r, rf in ((st.u, st.rhsx, st.rhsx_f), (st.v, st.rhsy, st.rhsy_f), (st.w, st.rhsz, st.rhsz_f)):
        f[k] = f[k] + p.dt * (tadv1 * r[k] + (1.0 - tadv1) * rf[k])
    st.w[0] = 0.0
    st.w[p.nz + 1] = 0.0
    return ops, st


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("grid", [dict(nx=32, ny=32, nz=32), dict(nx=256, ny=256, nz=4)])
def test_press_from_increment(gpu, grid, precision):
    """les_press_from_increment (the mixed step's pressure solve) against the
    oracle's press_stag_array on the same advanced state.  FP64: the same
    pressure to 1e-12 (the formulations differ only in rounding).  Mixed:
    FP32 inputs and transforms against the FP64 oracle on the unrounded
    state, 1e-5 -- the error of the path itself, the rounding of u* to FP32
    included (the direct formulation transforms that rounding divided by dt)."""
    p = O.Params(dt=2e-4, **grid)
    ops, st = _advance(p)
    les = _les(p, precision)
    gst = st.copy()
    if precision == "mixed":
        _round_f32(gst)
    mirror(les, gst)
    O.press_stag_array(ops, st, 1.5)
    les.press_from_increment(1.5)
    for name in ("p", "dpdx", "dpdy", "dpdz"):
        a, b = les.download(name), getattr(st, name)
        if name == "p":
            a, b = a[:-1], b[:-1]
        e = rel_err(a, b)
        assert e <= TOL[precision], (grid, precision, name, e)
    assert les.status() == 0
    les.close()
