"""Per-operator and multi-step parity of the CUDA library against the FP64
oracle, on identical seeded fields.

Tolerances (normwise relative, max|gpu - oracle| / max|oracle| per field,
BOGUS sentinels excluded): FP64 mode <= 1e-12, mixed precision (FP32 fields)
<= 1e-5 per operator.
"""
import numpy as np
import pytest

from oracle import les_oracle as O
from tests.helpers import field_errors, mirror, oracle_run, run_params, worst

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "mixed": 1e-5}


def _les(p, precision="fp64"):
    from new_repo_b200 import LES

    return LES(run_params(p), precision=precision)


def _pair(p, nsteps=3, precision="fp64", seed=0):
    ops, st = oracle_run(p, nsteps, seed)
    les = _les(p, precision)
    mirror(les, st)
    return ops, st, les


def _assert_close(les, st, tol, label):
    errs = field_errors(les, st)
    k, e = worst(errs)
    assert e <= tol, f"{label}: worst field {k} rel err {e:.3e} > {tol:.1e}; all: " + \
        ", ".join(f"{n}={v:.1e}" for n, v in sorted(errs.items(), key=lambda x: -x[1])[:6])


GRIDS = [dict(nx=32, ny=32, nz=32), dict(nx=64, ny=32, nz=16)]


@pytest.mark.parametrize("grid", GRIDS)
def test_grad_velocity_filt(gpu, grid):
    p = O.Params(**grid)
    ops, st, les = _pair(p)
    O.grad_velocity_filt(ops, st.v, st.dvdx, st.dvdy)
    les.grad_velocity_filt("v", "dvdx", "dvdy")
    _assert_close(les, st, TOL["fp64"], "grad_velocity_filt")


def test_single_mode_derivative_exact(gpu):
    """Known answer: d/dx sin(3x) = 3 cos(3x), d/dy cos(2y) = -2 sin(2y)."""
    p = O.Params(nx=32, ny=32, nz=4)
    les = _les(p)
    x = np.arange(p.nx) * p.dx
    y = np.arange(p.ny) * p.dy
    f = np.sin(3 * x)[None, None, :] + np.cos(2 * y)[None, :, None] + np.zeros((p.nz + 2, p.ny, p.nx))
    les.upload("u", f)
    les.grad_velocity_filt("u", "dudx", "dudy")
    dx = les.download("dudx")
    dy = les.download("dudy")
    assert np.abs(dx - 3 * np.cos(3 * x)[None, None, :]).max() < 1e-12
    assert np.abs(dy + 2 * np.sin(2 * y)[None, :, None]).max() < 1e-12


@pytest.mark.parametrize("grid", GRIDS)
def test_compute_vel_grad(gpu, grid):
    p = O.Params(**grid)
    ops, st, les = _pair(p)
    O.compute_vel_grad(ops, st)
    les.compute_vel_grad()
    _assert_close(les, st, TOL["fp64"], "compute_vel_grad")


@pytest.mark.parametrize("model", ["wall_filter", "wall_inst", "wall_homog"])
def test_wall_law(gpu, model):
    p = O.Params(nx=32, ny=32, nz=16, wall_model=model)
    ops, st, les = _pair(p)
    O.obukhov(ops, st)
    O.wallstress(ops, st)
    les.obukhov()
    les.wallstress()
    _assert_close(les, st, TOL["fp64"], f"wall law {model}")


@pytest.mark.parametrize("model", ["wall_inst", "wall_homog"])
def test_wall_law_model_argument(gpu, model):
    """obukhov(ustar_avg, wl_type) / wallstress(bc_u, bc_v, wl_type): the
    model passed per call (a state created with wall_filter) equals the
    oracle run with that model."""
    p = O.Params(nx=32, ny=32, nz=16, wall_model=model)
    ops, st, les = _pair(O.Params(nx=32, ny=32, nz=16, wall_model="wall_filter"))
    ops = O.Ops(p)
    O.obukhov(ops, st)
    O.wallstress(ops, st)
    les.obukhov(model)
    les.wallstress(model)
    _assert_close(les, st, TOL["fp64"], f"wall law {model} by argument")


@pytest.mark.parametrize("alpha", [2, 4])
def test_test_filter(gpu, alpha):
    from tests.helpers import rel_err

    p = O.Params(nx=32, ny=32, nz=16)
    ops, st, les = _pair(p)
    f = st.u.copy()
    les.upload("u_lag", f)
    O.test_filter(ops, f, ops.g_test if alpha == 2 else ops.g_test_test)
    les.test_filter("u_lag", alpha)
    assert rel_err(les.download("u_lag")[1:], f[1:]) <= TOL["fp64"]


@pytest.mark.parametrize("dealias", ["padd", "trunc"])
@pytest.mark.parametrize("grid", GRIDS)
def test_dealias_convec(gpu, dealias, grid):
    p = O.Params(dealias=dealias, **grid)
    ops, st, les = _pair(p)
    O.compute_dealias_convec(p, st, st.rhsx, st.rhsy, st.rhsz)
    les.compute_dealias_convec("rhsx", "rhsy", "rhsz")
    # the library's rhs store also moves rhs to rhs_f (compute_RHS_adv fusion);
    # compare the convective outputs only
    from tests.helpers import rel_err

    for n in ("rhsx", "rhsy", "rhsz"):
        e = rel_err(les.download(n), getattr(st, n))
        assert e <= TOL["fp64"], f"{dealias} {n}: {e:.3e}"


@pytest.mark.parametrize("stag", [True, False])
def test_div_stress(gpu, stag):
    p = O.Params(nx=32, ny=32, nz=16)
    ops, st, les = _pair(p)
    if stag:
        O.div_stress(ops, st.rhsx, st.txx, st.txy, st.txz, True)
        les.div_stress("rhsx", "txx", "txy", "txz", True)
    else:
        bot, top = O.div_stress(ops, st.rhsz, st.txz, st.tyz, st.tzz, False, want_layers=True)
        st.bottom_wk_press[:] = bot
        st.top_wk_press[:] = top
        les.div_stress("rhsz", "txz", "tyz", "tzz", False)
    _assert_close(les, st, TOL["fp64"], "div_stress")


@pytest.mark.parametrize("grid", GRIDS)
def test_compute_rhs_adv(gpu, grid):
    p = O.Params(**grid)
    ops, st, les = _pair(p)
    O.compute_rhs_adv(ops, st)
    les.compute_RHS_adv()
    _assert_close(les, st, TOL["fp64"], "compute_RHS_adv")


def _advance_to_pressure(ops, st, tadv1):
    """The part of LES_engine.f90:189-283 that precedes press_stag_array."""
    p = ops.p
    st.jt_total += 1
    O.obukhov(ops, st)
    O.wallstress(ops, st)
    O.compute_vel_grad(ops, st)
    O.sgs_stress(ops, st, st.jt_total, st.jt_total)
    O.compute_rhs_adv(ops, st)
    k = slice(1, p.nz + 1)
    tadv2 = 1.0 - tadv1
    for f, r, rf in ((st.u, st.rhsx, st.rhsx_f), (st.v, st.rhsy, st.rhsy_f), (st.w, st.rhsz, st.rhsz_f)):
        f[k] = f[k] + p.dt * (tadv1 * r[k] + tadv2 * rf[k])
    st.w[0] = 0.0
    st.w[p.nz + 1] = 0.0


@pytest.mark.parametrize("tadv1", [1.0, 1.5])
@pytest.mark.parametrize("grid", GRIDS)
def test_press_stag_array(gpu, grid, tadv1):
    """Pressure solve on the intermediate velocity u* of an AB2 advance."""
    p = O.Params(**grid)
    ops, st = oracle_run(p, 3)
    _advance_to_pressure(ops, st, tadv1)
    les = _les(p)
    mirror(les, st)
    O.press_stag_array(ops, st, tadv1)
    les.press_stag_array(tadv1)
    _assert_close(les, st, TOL["fp64"], "press_stag_array")


@pytest.mark.parametrize("model,nsteps", [("cst_Smag", 2), ("dyn_LagScaleDep", 2), ("dyn_LagScaleDep", 4),
                                          ("dyn_LagScaleDep", 9), ("dyn_Smag", 4)])
def test_sgs_stress(gpu, model, nsteps):
    """nsteps before the call: LASD at jtt=3 (accumulate only), jtt=5 (F
    initialisation), jtt=10 (Lagrangian interpolation + update)."""
    p = O.Params(nx=32, ny=32, nz=16, sgs_model=model)
    ops, st, les = _pair(p, nsteps)
    # sgs_stress consumes this step's gradients
    if p.lbc_special == "wall_law":
        O.obukhov(ops, st)
        O.wallstress(ops, st)
    O.compute_vel_grad(ops, st)
    mirror(les, st)
    jtt = nsteps + 1
    O.sgs_stress(ops, st, jtt, jtt)
    les.sgs_stress(jtt, jtt)
    _assert_close(les, st, TOL["fp64"], f"sgs_stress {model} jtt={jtt}")


@pytest.mark.parametrize("lag_halo", ["reference1x1", "periodic"])
def test_lagrangian_interpolation_halo(gpu, lag_halo):
    p = O.Params(nx=32, ny=32, nz=16, lag_halo=lag_halo)
    ops, st, les = _pair(p, 9)
    O.obukhov(ops, st)
    O.wallstress(ops, st)
    O.compute_vel_grad(ops, st)
    mirror(les, st)
    O.sgs_stress(ops, st, 10, 10)
    les.sgs_stress(10, 10)
    _assert_close(les, st, TOL["fp64"], f"LASD update {lag_halo}")


@pytest.mark.parametrize("cfg", [dict(nx=32, ny=32, nz=32), dict(nx=32, ny=32, nz=32, dealias="trunc"),
                                 dict(nx=32, ny=32, nz=32, dealias="trunc", sgs_model="cst_Smag"),
                                 dict(nx=64, ny=32, nz=16, sgs_model="cst_Smag")])
def test_ten_step_horizon(gpu, cfg):
    """10 full time steps from the same initial fields (LASD updates at 5, 10)."""
    p = O.Params(**cfg)
    ops, st = oracle_run(p, 0)
    les = _les(p)
    u, v, w = O.log_law_fields(p, seed=0)
    les.set_initial_conditions(u, v, w)
    for n in range(10):
        d_o = O.les_step(ops, st)
        les.step()
        d_g = les.diagnostics()
        assert np.allclose(d_g, d_o, rtol=1e-9, atol=1e-13), (n, d_g, d_o)
    errs = field_errors(les, st)
    # The reference rounds cs_opt2, beta, F_LM, F_QN to REAL(4)
    # (compute_LagScaleDep.f90:624-690): a 1e-16 difference in their FP64
    # inputs can move one point by one float ulp (6e-8), and that difference
    # reaches nu_t, tau and the rhs on the following steps (and u, v, w a
    # factor dt later).  Stated 10-step tolerances:
    #   SGS fields and rhs: <= 5e-7 (float-ulp propagation),
    #   u, v, w, p and their gradients: <= 1e-10.
    sgs = {"cs_opt2", "beta", "F_LM", "F_QN", "F_MM", "F_NN", "nu_t", "txx", "txy", "txz", "tyy", "tyz", "tzz",
           "rhsx", "rhsy", "rhsz", "rhsx_f", "rhsy_f", "rhsz_f", "bottom_wk_press", "top_wk_press"}
    e32 = max(errs[n] for n in sgs)
    k, e = worst({n: v for n, v in errs.items() if n not in sgs})
    # when one of those REAL(4) roundings did flip (cs_opt2 off by a float
    # ulp), its effect reaches the resolved fields at ~1e-9; otherwise the
    # FP64 bar holds
    flipped = errs["cs_opt2"] > 1e-12
    assert e <= (1e-8 if flipped else 1e-10), f"10-step worst field {k}: {e:.3e} (cs flip: {flipped})"
    assert e32 <= 5e-7, f"10-step SGS/rhs fields: {e32:.3e}"
    assert les.status() == 0


def test_initial_conditions_match(gpu):
    p = O.Params(nx=32, ny=32, nz=16)
    st = O.make_state(p)
    les = _les(p)
    les.set_initial_conditions(*O.log_law_fields(p, seed=0))
    errs = field_errors(les, st)
    assert worst(errs)[1] == 0.0


def _round_state_f32(st):
    """Identical inputs for the FP32 path: the oracle state rounded to FP32."""
    for n in O.FIELDS:
        a = getattr(st, n)
        a[:] = a.astype(np.float32).astype(np.float64)
    for n in ("lbc_u", "lbc_v", "lbc_w", "ubc_u", "ubc_v", "ubc_w", "bottom_wk_press", "top_wk_press",
              "lbc_z0", "u_star_avg"):
        a = getattr(st, n)
        a[:] = a.astype(np.float32).astype(np.float64)


@pytest.mark.parametrize("op", ["grad", "conv", "div", "press", "sgs"])
def test_mixed_precision_operators(gpu, op):
    """FP32 fields (FP64 tridiagonal pressure solve): per-operator error <= 1e-5
    against the FP64 oracle applied to the same FP32-representable inputs."""
    from tests.helpers import rel_err

    p = O.Params(nx=32, ny=32, nz=32)
    ops, st = oracle_run(p, 9)
    _round_state_f32(st)
    les = _les(p, "mixed")
    mirror(les, st)

    if op == "grad":
        O.compute_vel_grad(ops, st)
        les.compute_vel_grad()
        names = ["u", "v", "w", "dudx", "dudy", "dudz", "dvdx", "dvdy", "dvdz", "dwdx", "dwdy", "dwdz"]
    elif op == "conv":
        O.compute_dealias_convec(p, st, st.rhsx, st.rhsy, st.rhsz)
        les.compute_dealias_convec()
        names = ["rhsx", "rhsy", "rhsz"]
    elif op == "div":
        O.div_stress(ops, st.rhsx, st.txx, st.txy, st.txz, True)
        les.div_stress("rhsx", "txx", "txy", "txz", True)
        names = ["rhsx"]
    elif op == "press":
        _advance_to_pressure(ops, st, 1.5)
        _round_state_f32(st)
        mirror(les, st)
        O.press_stag_array(ops, st, 1.5)
        les.press_stag_array(1.5)
        names = ["p", "dpdx", "dpdy", "dpdz"]
    else:
        O.obukhov(ops, st)
        O.wallstress(ops, st)
        O.compute_vel_grad(ops, st)
        _round_state_f32(st)
        mirror(les, st)
        O.sgs_stress(ops, st, 10, 10)
        les.sgs_stress(10, 10)
        names = ["cs_opt2", "nu_t", "txx", "txy", "txz", "tyy", "tyz", "tzz"]
    for n in names:
        a = les.download(n)
        b = getattr(st, n)
        if n == "p":  # p(nz+1) is the BOGUS sentinel; compare the solved levels
            a, b = a[:-1], b[:-1]
        e = rel_err(a, b)
        assert e <= TOL["mixed"], f"mixed {op} {n}: {e:.3e}"
