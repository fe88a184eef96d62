"""Host-side mirror of the reference's LES module interface, driving the
B200 library through its C ABI.

The Fortran reference exposes module subroutines that act on module-global
arrays (``src/system.f90:21-43``); ``LES`` keeps those arrays in HBM and
offers the same entry points under the same names:

=====================================  ==========================================
reference (file:line)                  here
=====================================  ==========================================
read_parameters  parameters_IO.f90:128 ``RunParams`` / ``read_namelist``
create_system + *_init                 ``LES(params)``
set_initial_conditions ('files')       ``LES.set_initial_conditions``
initial_conditions.f90:130-212
grad_velocity_filt                     ``LES.grad_velocity_filt``
compute_derivatives.f90:94
ddz_uv / ddz_w  :375 / :413            ``LES.ddz_uv`` / ``LES.ddz_w``
div_stress  :464                       ``LES.div_stress``
compute_dealias_convec                 ``LES.compute_dealias_convec``
compute_convective_padd.f90:115
press_stag_array compute_pressure:116  ``LES.press_stag_array``
obukhov / wallstress                   ``LES.obukhov`` / ``LES.wallstress``
compute_wall_law.f90:198 / :107
sgs_stress compute_sgs.f90:105         ``LES.sgs_stress``
test_filter testfilter.f90:144         ``LES.test_filter``
set_bc boundary_condition_mpi.f90:33   ``LES.set_bc``
compute_vel_grad LES_engine.f90:449    ``LES.compute_vel_grad``
compute_RHS_adv LES_engine.f90:509     ``LES.compute_RHS_adv``
time loop body LES_engine.f90:189-360  ``LES.step``
compute_running_diagnistics            ``LES.diagnostics``
running_diagnostics.f90:80
checkpoint_out / checkpoint_in         ``LES.checkpoint_out`` / ``checkpoint_in``
IO_checkpoint.f90:53-256
io_stat_init / io_stat_averages        ``LES.stat_init`` / ``LES.stat_averages``
IO_statistics.f90:40 / :265
io_stat_spectra  IO_statistics:566     ``LES.stat_spectra``
tke_budget_init / compute_tke_budget   ``LES.tke_init`` / ``LES.tke_budget``
tke_budget1D.f90:61 / :209
=====================================  ==========================================

Errors: the reference aborts through ``decomp_2d_abort(code, msg)``; here a
nonzero library status raises ``LesError`` carrying the same code
(1 invalid option, 3 out of memory, 9 numerical failure, 22 I/O).
"""
from __future__ import annotations

import copy
import ctypes as C
import math
import re
from dataclasses import dataclass, field, replace
from pathlib import Path

import numpy as np

from . import capi
from .capi import FIELD_ID, PLANE_ID, LesError, LesParams, check

PI = 3.1415926535897932384626433  # parameters_IO.f90:42
KVONK = 0.4


@dataclass
class RunParams:
    """Namelist parameters (parameters_IO.f90:151-166) and the derived sizes of
    read_parameters (:238-277)."""

    nx: int = 32
    ny: int = 32
    nz: int = 32
    dt: float = 2e-4
    dim_dt_flag: bool = False
    xy_pi: bool = True
    lx_in: float = 2.0
    ly_in: float = 2.0
    lz_in: float = 1.0
    zi: float = 1.0
    u_scale: float = 1.0
    lbc_dz0: float = 1e-4
    pfx: float = 1.0
    pfy: float = 0.0
    cs0: float = 0.16
    sgs_model: str = "dyn_LagScaleDep"
    cs_count: int = 5
    dyn_init: int = 5
    lbc_special: str = "wall_law"
    wall_model: str = "wall_filter"
    dealias: str = "padd"
    lag_halo: str = "reference1x1"
    # output_param (parameters_IO.f90:103-111,153-157): post-step statistics
    out_path: str = "./"
    stat_flag: bool = False
    start_stats: int = 0
    running_period: int = 1000
    tke_flag: bool = False
    start_tke: int = 0
    tke_period: int = 100
    spectra_flag: bool = False
    # LES_engine.f90:81 (a parameter there): check_NaN every nan_check steps
    nan_check: int = 20

    lx: float = field(init=False, default=0.0)
    ly: float = field(init=False, default=0.0)
    lz: float = field(init=False, default=0.0)
    dx: float = field(init=False, default=0.0)
    dy: float = field(init=False, default=0.0)
    dz: float = field(init=False, default=0.0)
    z0: float = field(init=False, default=0.0)
    dt_nd: float = field(init=False, default=0.0)

    def __post_init__(self):
        self.derive()

    def derive(self) -> "RunParams":
        lx, ly, lz = self.lx_in, self.ly_in, self.lz_in
        if self.xy_pi:
            lx = lx * PI
            ly = ly * PI
        self.lx, self.ly, self.lz = lx / self.zi, ly / self.zi, lz / self.zi
        self.dt_nd = self.dt * self.u_scale / self.zi if self.dim_dt_flag else self.dt
        self.dx = self.lx / float(self.nx)
        self.dy = self.ly / float(self.ny)
        self.dz = self.lz / float(self.nz)
        self.z0 = self.lbc_dz0 / self.zi
        return self

    def with_(self, **kw) -> "RunParams":
        return replace(self, **kw).derive()

    def to_c(self, precision: str = "fp64", device: int = 0) -> LesParams:
        for name, table, val in (("sgs_model", capi.SGS_MODELS, self.sgs_model),
                                 ("wall_model", capi.WALL_MODELS, self.wall_model),
                                 ("dealias", capi.DEALIAS, self.dealias),
                                 ("lag_halo", capi.LAG_HALO, self.lag_halo),
                                 ("precision", capi.PRECISION, precision)):
            if val not in table:
                raise LesError(capi.LES_ERR_INVALID, f"Invalid {name}: {val!r}")
        return LesParams(self.nx, self.ny, self.nz, self.dt_nd, self.lx, self.ly, self.lz, self.z0,
                         self.pfx, self.pfy, self.cs0, capi.SGS_MODELS[self.sgs_model], self.cs_count,
                         self.dyn_init, 1 if self.lbc_special == "wall_law" else 0,
                         capi.WALL_MODELS[self.wall_model], capi.DEALIAS[self.dealias],
                         capi.LAG_HALO[self.lag_halo], capi.PRECISION[precision], device)


_NML_KEYS = {"p_on_y", "p_on_z", "nx", "ny", "nz", "nt", "dt", "dim_dt_flag", "restart_flag", "xy_pi", "lx",
             "ly", "lz", "u_scale", "zi", "lbc_dz0", "re", "pfx", "pfy", "cs0", "sgs_model", "cs_count",
             "dyn_init", "lbc_special", "wall_model",
             "out_path", "stat_flag", "start_stats", "running_period", "tke_flag", "start_tke", "tke_period",
             "spectra_flag"}


def _namelist_values(text: str) -> dict:
    """key = value pairs of a Fortran namelist (keys lower-cased; logicals,
    integers, reals with d/e exponents and quoted strings)."""
    raw = {}
    for m in re.finditer(r"(\w+)\s*=\s*('[^']*'|\"[^\"]*\"|[^\s,/]+)", text):
        key, val = m.group(1).lower(), m.group(2).strip()
        if val[0] in "'\"":
            v = val[1:-1]
        elif val.lower() in (".true.", "t", ".t."):
            v = True
        elif val.lower() in (".false.", "f", ".f."):
            v = False
        else:
            try:
                v = int(val)
            except ValueError:
                v = float(val.lower().replace("d", "e"))
        raw[key] = v
    return raw


def read_namelist(path: str | Path) -> tuple[RunParams, dict]:
    """Parse a ``parameters.nlst`` (parameters_IO.f90:151-234) into RunParams.

    Returns (params, raw) where raw holds every key=value found.  Raises
    LesError(22) when the file cannot be read, like the reference's
    MPI_Abort(22) (parameters_IO.f90:173-234)."""
    try:
        text = Path(path).read_text()
    except OSError as e:
        raise LesError(capi.LES_ERR_IO, f"Could not open {path} for reading ({e})") from e
    raw = _namelist_values(text)
    kw = dict(nx=raw.get("nx", 32), ny=raw.get("ny", 32), nz=raw.get("nz", 32), dt=float(raw.get("dt", 2e-4)),
              dim_dt_flag=bool(raw.get("dim_dt_flag", False)), xy_pi=bool(raw.get("xy_pi", True)),
              lx_in=float(raw.get("lx", 2.0)), ly_in=float(raw.get("ly", 2.0)), lz_in=float(raw.get("lz", 1.0)),
              zi=float(raw.get("zi", 1.0)), u_scale=float(raw.get("u_scale", 1.0)),
              lbc_dz0=float(raw.get("lbc_dz0", 1e-4)), pfx=float(raw.get("pfx", 1.0)),
              pfy=float(raw.get("pfy", 0.0)), cs0=float(raw.get("cs0", 0.16)),
              sgs_model=str(raw.get("sgs_model", "cst_Smag")), cs_count=int(raw.get("cs_count", 5)),
              dyn_init=int(raw.get("dyn_init", 1500)), lbc_special=str(raw.get("lbc_special", "std")),
              wall_model=str(raw.get("wall_model", "wall_filter")))
    for key, typ in (("out_path", str), ("stat_flag", bool), ("start_stats", int), ("running_period", int),
                     ("tke_flag", bool), ("start_tke", int), ("tke_period", int), ("spectra_flag", bool)):
        if key in raw:
            kw[key] = typ(raw[key])
    return RunParams(**kw), raw


def write_parameters_restart(path: str | Path, p: RunParams, jt_total: int, lagran_init: bool) -> None:
    """``parameters_restart.nlst`` as write_parameters_restart writes it
    (parameters_IO.f90:333-369): the restart_param namelist of one rank."""
    t = "T" if lagran_init else "F"
    text = (f"&RESTART_PARAM\n P_ON_Y_F=1,\n P_ON_Z_F=1,\n NX_F={p.nx},\n NY_F={p.ny},\n NZ_F={p.nz},\n"
            f" JT_TOTAL={int(jt_total)},\n DYN_INIT={int(p.dyn_init)},\n LAGRAN_INIT={t},\n"
            f" SGS_MODEL='{p.sgs_model}',\n /\n")
    try:
        Path(path).write_text(text)
    except OSError as e:
        raise LesError(capi.LES_ERR_IO, f"Could not open {path} for writing ({e})") from e


def read_parameters_restart(path: str | Path, p: RunParams) -> dict:
    """read_parameters_restart (parameters_IO.f90:380-435): jt_total,
    dyn_init, Lagran_init and sgs_model of a restart; LesError(22) when the
    file cannot be read, LesError(1) when the grid differs from ``p``."""
    try:
        raw = _namelist_values(Path(path).read_text())
    except OSError as e:
        raise LesError(capi.LES_ERR_IO, f"Could not open {path} for reading ({e})") from e
    need = ("nx_f", "ny_f", "nz_f", "jt_total", "lagran_init")
    if any(k not in raw for k in need):
        raise LesError(capi.LES_ERR_IO, f"Error in namelist restart_param of {path}")
    if (raw["nx_f"], raw["ny_f"], raw["nz_f"]) != (p.nx, p.ny, p.nz):
        raise LesError(capi.LES_ERR_INVALID, "[Restart error] invalid restart parameters")
    return {"jt_total": int(raw["jt_total"]), "dyn_init": int(raw.get("dyn_init", p.dyn_init)),
            "lagran_init": bool(raw["lagran_init"]), "sgs_model": str(raw.get("sgs_model", p.sgs_model))}


def log_law_noise(p: RunParams, seed: int = 0, amp: float = 0.1):
    """Synthetic initial velocity (nz, ny, nx): u = ln(z/z0)/kappa at uvp heights
    z = (k-1/2) dz (initial_conditions.f90:101-117 with u_star = 1) plus
    uniform noise in [-amp, amp) from a counter-based hash of
    (seed, field, index) (splitmix64).  The reference's own ran3 noise is not
    reproduced; fields are handed over through the ic_type='files' path."""
    z = (np.arange(1, p.nz + 1) - 0.5) * p.dz
    arg = (1.0 / KVONK) * np.log(z / p.z0)
    shape = (p.nz, p.ny, p.nx)
    u = np.broadcast_to(arg[:, None, None], shape).copy()
    v = np.zeros(shape)
    w = np.zeros(shape)
    for fid, a in enumerate((u, v, w)):
        a += amp * _hash_uniform(seed, fid, shape)
    return u, v, w


def scalar_linear_noise(p: RunParams, seed: int = 0, amp: float = 0.01, gradient: float = 1.0):
    """Passive-scalar initial field (nz, ny, nx): gradient * z at the uvp
    heights plus uniform noise in [-amp, amp) (the velocity's hash, stream 3)."""
    z = (np.arange(1, p.nz + 1) - 0.5) * p.dz
    th = gradient * z[:, None, None] + np.zeros((p.nz, p.ny, p.nx))
    return th + amp * _hash_uniform(seed, 3, th.shape)


def inversion_noise(p: RunParams, seed: int = 0, z_inv: float = 0.5, lapse: float = 10.0, amp: float = 0.1,
                    z_noise: float = 0.1):
    """Convective-boundary-layer temperature as the departure from theta_0
    (nz, ny, nx): 0 up to z_inv, lapse * (z - z_inv) above (0.01 K/m with
    z_i = 1000 m is 10 K per unit height), uniform noise in [-amp, amp) K
    below z_noise (hash stream 3)."""
    z = (np.arange(1, p.nz + 1) - 0.5) * p.dz
    base = np.where(z > z_inv, lapse * (z - z_inv), 0.0)
    th = base[:, None, None] + np.zeros((p.nz, p.ny, p.nx))
    noise = amp * _hash_uniform(seed, 3, th.shape)
    return th + np.where((z < z_noise)[:, None, None], noise, 0.0)


def _hash_uniform(seed: int, fid: int, shape):
    n = int(np.prod(shape))
    x = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = x + np.uint64((seed * 1000003 + fid * 7919 + 1) & 0xFFFFFFFFFFFFFFFF) * np.uint64(0x9E3779B97F4A7C15)
        z = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    u01 = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    return (2.0 * u01 - 1.0).reshape(shape)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class LES:
    """One device-resident LES state on one GPU."""

    def __init__(self, params: RunParams, precision: str = "fp64", device: int = 0):
        self.lib = capi.load()
        self.params = copy.copy(params)  # set_sgs_model changes this instance's copy only
        self.precision = precision
        self._cp = params.to_c(precision, device)
        h = C.c_void_p()
        check(self.lib.les_create(C.byref(self._cp), C.byref(h)))
        self._h = h
        self.jt_total = 0
        self.jt = 0
        # io_stat_init / tke_budget_init when their flags are on (LES_engine.f90:149-150)
        if self.params.stat_flag:
            self.stat_init()
        if self.params.tke_flag:
            self.tke_init()

    # ------------------------------------------------------------- lifetime
    def close(self):
        if getattr(self, "_h", None):
            self.lib.les_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------- data movement
    @property
    def shape(self):
        p = self.params
        return (p.nz + 2, p.ny, p.nx)

    def _fid(self, f) -> int:
        if isinstance(f, str):
            if f not in FIELD_ID:
                raise LesError(capi.LES_ERR_INVALID, f"unknown field {f!r}")
            return FIELD_ID[f]
        return int(f)

    def upload(self, name, arr, k0: int = 0, k1: int | None = None):
        k1 = self.params.nz + 1 if k1 is None else k1
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.size != (k1 - k0 + 1) * self.params.ny * self.params.nx:
            raise LesError(capi.LES_ERR_INVALID, "array size does not match the level range")
        check(self.lib.les_upload(self._h, self._fid(name), _dptr(a), k0, k1))

    def download(self, name, k0: int = 0, k1: int | None = None) -> np.ndarray:
        k1 = self.params.nz + 1 if k1 is None else k1
        out = np.empty((k1 - k0 + 1, self.params.ny, self.params.nx))
        check(self.lib.les_download(self._h, self._fid(name), _dptr(out), k0, k1))
        return out

    def upload_plane(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        check(self.lib.les_upload_plane(self._h, PLANE_ID[name], _dptr(a)))

    def download_plane(self, name) -> np.ndarray:
        out = np.empty((self.params.ny, self.params.nx))
        check(self.lib.les_download_plane(self._h, PLANE_ID[name], _dptr(out)))
        return out

    # ------------------------------------------------- scalar and forcing
    def scalar_init(self, surface_flux: float = 0.0, top_gradient: float = 0.0, buoyancy: float = 0.0,
                    pr_t: float = 0.4, sgs: str = "dynamic"):
        """scalars_module_init (compute_scalars.f90:40-57): theta on uvp nodes
        with the SGS flux of the constant- or dynamic-Prandtl model, a wall
        flux, a lid gradient and (buoyancy = g/theta_0 != 0) buoyancy in the
        w equation; see les_scalar_init in lesgpu.h."""
        if sgs not in capi.SCALAR_SGS:
            raise LesError(capi.LES_ERR_INVALID, f"Invalid scalar SGS model {sgs!r}")
        sp = capi.ScalarParams(float(surface_flux), float(top_gradient), float(buoyancy), float(pr_t),
                               capi.SCALAR_SGS[sgs])
        check(self.lib.les_scalar_init(self._h, C.byref(sp)))

    def scalar_set_initial(self, theta):
        """theta (nz, ny, nx) on levels 1..nz; the ghost values follow."""
        a = np.ascontiguousarray(theta, dtype=np.float64)
        p = self.params
        if a.shape != (p.nz, p.ny, p.nx):
            raise LesError(capi.LES_ERR_INVALID, "theta must be (nz, ny, nx)")
        check(self.lib.les_scalar_set_initial(self._h, _dptr(a)))

    def scalar_kappa(self) -> np.ndarray:
        """Cs^2/Pr_t per level 0..nz+1 of the dynamic Prandtl model (0 for the constant one)."""
        out = np.zeros(self.params.nz + 2)
        check(self.lib.les_scalar_kappa(self._h, _dptr(out), out.size))
        return out

    def sponge_init(self, layer_fraction: float):
        """sponge_damping_init (sponge_damping.f90:42-101, no zeroing): damping
        above layer_fraction * lz, applied at the end of compute_RHS_adv."""
        check(self.lib.les_sponge_init(self._h, float(layer_fraction)))

    def set_cs2_max(self, cs2_max: float):
        """Upper clip of the dynamic Cs^2 (0 = none, the reference's behaviour)."""
        check(self.lib.les_set_cs2_max(self._h, float(cs2_max)))

    def set_coriolis(self, coriol: float, ug: float = 0.0, vg: float = 0.0):
        """Coriolis forcing of compute_RHS_adv (LES_engine.f90:553-561)."""
        check(self.lib.les_set_coriolis(self._h, float(coriol), float(ug), float(vg)))

    def set_initial_conditions(self, u, v, w):
        a = [np.ascontiguousarray(x, dtype=np.float64) for x in (u, v, w)]
        check(self.lib.les_set_initial_conditions(self._h, *map(_dptr, a)))

    def set_bc_types(self, lbc=(2, 2, 1), ubc=(2, 2, 1)):
        la = (C.c_int * 3)(*lbc)
        ua = (C.c_int * 3)(*ubc)
        check(self.lib.les_set_bc_types(self._h, la, ua))

    @property
    def f_coeff_init(self) -> bool:
        v = C.c_int()
        check(self.lib.les_get_lagrangian_init(self._h, C.byref(v)))
        return bool(v.value)

    @f_coeff_init.setter
    def f_coeff_init(self, val: bool):
        check(self.lib.les_set_lagrangian_init(self._h, 1 if val else 0))

    # -------------------------------------------------- module entry points
    def grad_velocity_filt(self, f, dfdx, dfdy):
        check(self.lib.les_grad_velocity_filt(self._h, self._fid(f), self._fid(dfdx), self._fid(dfdy)))

    def ddz_uv(self, dfdz, f):
        check(self.lib.les_ddz_uv(self._h, self._fid(dfdz), self._fid(f)))

    def ddz_w(self, dfdz, f):
        check(self.lib.les_ddz_w(self._h, self._fid(dfdz), self._fid(f)))

    def div_stress(self, rhs, tx, ty, tz, stag: bool):
        check(self.lib.les_div_stress(self._h, *(self._fid(x) for x in (rhs, tx, ty, tz)), 1 if stag else 0))

    def compute_dealias_convec(self, cx="rhsx", cy="rhsy", cz="rhsz"):
        check(self.lib.les_compute_dealias_convec(self._h, self._fid(cx), self._fid(cy), self._fid(cz)))

    def press_stag_array(self, tadv1: float):
        check(self.lib.les_press_stag_array(self._h, float(tadv1)))

    def set_pressure_slabs(self, nslabs: int):
        """Solve the pressure systems by the partition method over nslabs
        z-slabs (the decomposed solve emulated on one GPU); 1 = single sweep."""
        check(self.lib.les_set_pressure_slabs(self._h, int(nslabs)))

    def press_from_increment(self, tadv1: float, tadv2: float | None = None):
        """press_stag_array in increment form for the state les_ab2_advance
        left (see les_press_from_increment in lesgpu.h)."""
        tadv2 = 1.0 - float(tadv1) if tadv2 is None else float(tadv2)
        check(self.lib.les_press_from_increment(self._h, float(tadv1), tadv2))

    def set_wall_model(self, wl_type: str):
        """The wl_type argument of obukhov / wallstress ('wall_filter',
        'wall_inst', 'wall_homog'), kept for later calls and les_step."""
        if wl_type not in capi.WALL_MODELS:
            raise LesError(capi.LES_ERR_INVALID, f"Invalid wall model: {wl_type!r}")
        check(self.lib.les_set_wall_model(self._h, capi.WALL_MODELS[wl_type]))
        self.params = replace(self.params, wall_model=wl_type)

    def obukhov(self, wl_type: str | None = None):
        """compute_wall_law.f90:198-254 obukhov(u_star_avg, wl_type)."""
        if wl_type is not None:
            self.set_wall_model(wl_type)
        check(self.lib.les_obukhov(self._h))

    def wallstress(self, wl_type: str | None = None):
        """compute_wall_law.f90:107-185 wallstress(lbc_u, lbc_v, wl_type)."""
        if wl_type is not None:
            self.set_wall_model(wl_type)
        check(self.lib.les_wallstress(self._h))

    def sgs_stress(self, jt: int, jtt: int):
        check(self.lib.les_sgs_stress(self._h, int(jt), int(jtt)))

    def test_filter(self, f, alpha: int = 2):
        check(self.lib.les_test_filter(self._h, self._fid(f), int(alpha)))

    def set_bc(self):
        check(self.lib.les_set_bc(self._h))

    def compute_vel_grad(self):
        check(self.lib.les_compute_vel_grad(self._h))

    def compute_RHS_adv(self):
        check(self.lib.les_compute_rhs_adv(self._h))

    def ab2_advance(self, tadv1: float, tadv2: float):
        check(self.lib.les_ab2_advance(self._h, float(tadv1), float(tadv2)))

    def projection(self, tadv1: float):
        check(self.lib.les_projection(self._h, float(tadv1)))

    def step(self, n: int = 1):
        """Advance n time steps (the LES_engine.f90:189-360 loop body), each
        followed by the statistics its output flags ask for (:366-380)."""
        p = self.params
        for _ in range(n):
            self.jt += 1
            self.jt_total += 1
            check(self.lib.les_step(self._h, self.jt, self.jt_total))
            if p.nan_check > 0 and self.jt % p.nan_check == 0:  # LES_engine.f90:363-365
                self.check_status()
            if p.stat_flag and self.jt_total > p.start_stats:
                self.stat_averages()
            if p.spectra_flag:
                self.stat_spectra()
            if p.tke_flag and self.jt_total > p.start_tke:
                self.tke_budget()

    # --------------------------------------------------------------- statistics
    def stat_init(self):
        """io_stat_init (IO_statistics.f90:40-250): running sums allocated and zeroed."""
        check(self.lib.les_stat_init(self._h))

    def stat_averages(self, jt: int | None = None, jt_total: int | None = None):
        """io_stat_averages(jt, jt_total) (IO_statistics.f90:265-518): add the
        state to the running sums; RAV_<jt_total>_{info.txt,2D.dat,3D.dat}
        under out_path every running_period steps after start_stats."""
        p = self.params
        jt = self.jt if jt is None else int(jt)
        jt_total = self.jt_total if jt_total is None else int(jt_total)
        check(self.lib.les_stat_averages(self._h, jt, jt_total, int(p.start_stats), int(p.running_period),
                                         p.out_path.encode()))

    def stat_sums(self, name: str) -> np.ndarray:
        """The running sum ``name`` (STAT_NAMES order, or "ustar") as
        (nz, ny, nx) / (ny, nx) FP64."""
        p = self.params
        if name == "ustar":
            out = np.empty((p.ny, p.nx))
            idx = len(capi.STAT_NAMES)
        else:
            if name not in capi.STAT_NAMES:
                raise LesError(capi.LES_ERR_INVALID, f"unknown statistic {name!r}")
            out = np.empty((p.nz, p.ny, p.nx))
            idx = capi.STAT_NAMES.index(name)
        check(self.lib.les_stat_sums(self._h, idx, _dptr(out)))
        return out

    def stat_iterations(self) -> int:
        v = C.c_int()
        check(self.lib.les_stat_iterations(self._h, C.byref(v)))
        return int(v.value)

    def stat_spectra(self, jt: int | None = None, jt_total: int | None = None):
        """io_stat_spectra (IO_statistics.f90:566-620)."""
        jt = self.jt if jt is None else int(jt)
        jt_total = self.jt_total if jt_total is None else int(jt_total)
        check(self.lib.les_stat_spectra(self._h, jt, jt_total, self.params.out_path.encode()))

    def tke_init(self):
        """tke_budget_init (tke_budget1D.f90:61-160): out_path/ta1_profiles/,
        61 zeroed profiles, record counter 1."""
        check(self.lib.les_tke_init(self._h, self.params.out_path.encode()))

    def tke_budget(self, jt: int | None = None):
        """compute_tke_budget(jt) (tke_budget1D.f90:209-390)."""
        jt = self.jt if jt is None else int(jt)
        check(self.lib.les_tke_budget(self._h, jt, int(self.params.tke_period)))

    def tke_profiles(self) -> tuple[np.ndarray, int]:
        """(61, nz) running plane averages (TKE_NAMES order) and the next record number."""
        out = np.empty((len(capi.TKE_NAMES), self.params.nz))
        rec = C.c_int()
        check(self.lib.les_tke_sums(self._h, _dptr(out), C.byref(rec)))
        return out, int(rec.value)

    def diagnostics(self) -> tuple:
        """(cfl, mke, u_star, rms div u) of running_diagnostics.f90:148-305."""
        out = np.zeros(4)
        check(self.lib.les_diagnostics(self._h, _dptr(out)))
        return tuple(float(x) for x in out)

    def status(self) -> int:
        v = C.c_uint()
        check(self.lib.les_get_status(self._h, C.byref(v)))
        return int(v.value)

    def check_status(self) -> int:
        """check_NaN (LES_engine.f90:583-616) and the tridiagonal pivot abort
        (compute_pressure.f90:411-418): LesError(9) with the reference's
        message when either happened since the last read; otherwise the
        status bits (read and cleared)."""
        v = C.c_uint()
        check(self.lib.les_check_status(self._h, C.byref(v)))
        return int(v.value)

    def sync(self):
        check(self.lib.les_sync(self._h))

    def timers(self) -> dict:
        out = np.zeros(5)
        check(self.lib.les_timers(self._h, _dptr(out)))
        return dict(zip(("grad", "stress", "rhs", "press", "loop"), out.tolist()))

    # ------------------------------------------------------------ measurement
    def profile(self, enable: bool = True):
        check(self.lib.les_profile(self._h, 1 if enable else 0))

    def profile_report(self) -> dict:
        import json

        buf = C.create_string_buffer(1 << 20)
        check(self.lib.les_profile_report(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def launch_count(self) -> int:
        v = C.c_longlong()
        check(self.lib.les_launch_count(self._h, C.byref(v)))
        return int(v.value)

    def event_record(self, slot: int):
        check(self.lib.les_event_record(self._h, int(slot)))

    def event_elapsed(self, a: int, b: int) -> float:
        v = C.c_double()
        check(self.lib.les_event_elapsed(self._h, int(a), int(b), C.byref(v)))
        return float(v.value)

    def upload_async(self, name, pinned_ptr: int, k0: int = 0, k1: int | None = None):
        """Copy levels k0..k1 of a field from page-locked host memory (address)."""
        k1 = self.params.nz + 1 if k1 is None else k1
        check(self.lib.les_upload_async(self._h, self._fid(name), C.c_void_p(pinned_ptr), k0, k1))

    def download_async(self, name, pinned_ptr: int, k0: int = 0, k1: int | None = None):
        k1 = self.params.nz + 1 if k1 is None else k1
        check(self.lib.les_download_async(self._h, self._fid(name), C.c_void_p(pinned_ptr), k0, k1))

    def diagnostics_async(self, pinned_ptr: int):
        check(self.lib.les_diagnostics_async(self._h, C.c_void_p(pinned_ptr)))

    def step_host(self, u_ptr: int, v_ptr: int, w_ptr: int, diag_ptr: int | None = None, n: int = 1):
        """Advance n time steps with u, v, w held in host memory (addresses of
        FP64 arrays of shape (nz + 2, ny, nx), page-locked for the copies to
        overlap): each step copies them in, steps, and copies the new state
        and its diagnostics back (les_step_host).  Asynchronous like the
        C entry point: sync() before touching the arrays.  The status check
        and the statistics of step() follow at the same steps."""
        p = self.params
        d = C.c_void_p(diag_ptr) if diag_ptr else None
        for _ in range(n):
            self.jt += 1
            self.jt_total += 1
            check(self.lib.les_step_host(self._h, self.jt, self.jt_total, C.c_void_p(u_ptr), C.c_void_p(v_ptr),
                                         C.c_void_p(w_ptr), d))
            if p.nan_check > 0 and self.jt % p.nan_check == 0:
                self.check_status()
            if p.stat_flag and self.jt_total > p.start_stats:
                self.stat_averages()
            if p.spectra_flag:
                self.stat_spectra()
            if p.tke_flag and self.jt_total > p.start_tke:
                self.tke_budget()

    # ------------------------------------------------------ learned closure
    def set_precision(self, precision: str):
        """Move the state to the other precision ("fp64" / "mixed"): fields,
        planes, boundary-condition types and Lagrangian flags carry over."""
        if precision not in capi.PRECISION:
            raise LesError(capi.LES_ERR_INVALID, f"Invalid precision: {precision!r}")
        check(self.lib.les_set_precision(self._h, capi.PRECISION[precision]))
        self.precision = precision

    def set_sgs_model(self, name: str):
        """Switch the SGS closure ('cst_Smag', 'dyn_Smag', 'dyn_LagScaleDep', 'mlp')."""
        if name not in capi.SGS_MODELS:
            raise LesError(1, f"Invalid SGS model {name!r}")
        check(self.lib.les_set_sgs_model(self._h, capi.SGS_MODELS[name]))
        self.params.sgs_model = name

    def mlp_init(self, seed: int = 0):
        check(self.lib.les_mlp_init(self._h, int(seed) & 0xFFFFFFFF))

    def mlp_params(self) -> np.ndarray:
        """Flat float32 vector: the 4801 weights then the 34 feature/target statistics."""
        out = np.zeros(capi.MLP_NPARAM + capi.MLP_NSTATS, np.float32)
        check(self.lib.les_mlp_get_params(self._h, _fptr(out), out.size))
        return out

    def mlp_set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(self.lib.les_mlp_set_params(self._h, _fptr(p), p.size))

    def mlp_reset_data(self, cap: int):
        check(self.lib.les_mlp_reset_data(self._h, int(cap)))

    def mlp_collect(self, stride: int = 1, seed: int = 0, dense_levels: int = 0, wall_repeat: int = 1):
        """Append (features, log Cs^2) pairs of the current state: one point in
        ``stride``, every point of levels 1..dense_levels, the training pairs of
        levels 1 and 2 ``wall_repeat`` times.  Call right after consecutive
        dynamic-update steps (the first call only records the coefficient)."""
        check(self.lib.les_mlp_collect(self._h, int(stride), int(dense_levels), int(wall_repeat),
                                       int(seed) & 0xFFFFFFFF))

    def mlp_counts(self) -> tuple:
        out = (C.c_longlong * 2)()
        check(self.lib.les_mlp_counts(self._h, out))
        return int(out[0]), int(out[1])

    def mlp_fit_stats(self):
        check(self.lib.les_mlp_fit_stats(self._h))

    def mlp_train(self, epochs: int, tiles_per_step: int = 8, lr: float = 2e-3) -> tuple:
        """Adam epochs on the collected pairs; returns (last-batch loss per epoch, validation loss)."""
        losses = np.zeros(max(1, epochs))
        val = C.c_double()
        check(self.lib.les_mlp_train(self._h, int(epochs), int(tiles_per_step), float(lr), _dptr(losses),
                                     C.byref(val)))
        return losses[:epochs], float(val.value)

    def mlp_forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros(x.shape[0], np.float32)
        check(self.lib.les_mlp_forward(self._h, _fptr(x), x.shape[0], _fptr(y)))
        return y

    def mlp_grad(self, x, t) -> tuple:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(capi.MLP_NPARAM, np.float32)
        loss = np.zeros(1, np.float32)
        check(self.lib.les_mlp_grad(self._h, _fptr(x), _fptr(t), x.shape[0], _fptr(g), _fptr(loss)))
        return g, float(loss[0])

    def mlp_info(self) -> dict:
        out = np.zeros(12)
        check(self.lib.les_mlp_info(self._h, _dptr(out)))
        return {"check_rms_log_error": float(out[0]), "flagged_columns": int(out[1]), "updates": int(out[2]),
                "ready": bool(out[3]), "flagged_by_feature": [int(x) for x in out[4:12]]}

    def mlp_set_check_every(self, every: int):
        check(self.lib.les_mlp_set_check_every(self._h, int(every)))

    def mlp_check_profile(self) -> np.ndarray:
        """RMS log error of the closure against the dynamic procedure per level 1..nz+1 at the last check."""
        out = np.zeros(self.params.nz + 1)
        check(self.lib.les_mlp_check_profile(self._h, _dptr(out), out.size))
        return out

    def mlp_set_wall_levels(self, nlev: int):
        """Levels 1..nlev next to the wall keep the plain LASD procedure."""
        check(self.lib.les_mlp_set_wall_levels(self._h, int(nlev)))

    # ----------------------------------------------------------------- restart
    @property
    def lagran_init(self) -> bool:
        return self.f_coeff_init

    def checkpoint_out(self, directory: str | Path = ".", jt_total: int | None = None) -> Path:
        """checkpoint_out + write_parameters_restart (IO_checkpoint.f90:84-98,
        parameters_IO.f90:333-369): ``checkpoint_<jt_total:09d>`` (byte for
        byte the reference's file on one rank) and ``parameters_restart.nlst``."""
        jt_total = self.jt_total if jt_total is None else int(jt_total)
        d = Path(directory)
        path = d / f"checkpoint_{jt_total:09d}"
        check(self.lib.les_checkpoint_write(self._h, str(path).encode()))
        write_parameters_restart(d / "parameters_restart.nlst", self.params, jt_total, self.lagran_init)
        return path

    def checkpoint_in(self, directory: str | Path = ".") -> dict:
        """read_parameters_restart + checkpoint_in (LES_engine.f90:117-164):
        restores u, v, w, rhs, cs_opt2 (and the Lagrangian averages) and the
        step counter; the run continues with jt = 0, jt_total as saved."""
        d = Path(directory)
        rp = read_parameters_restart(d / "parameters_restart.nlst", self.params)
        path = d / f"checkpoint_{rp['jt_total']:09d}"
        check(self.lib.les_checkpoint_read(self._h, str(path).encode(), 1 if rp["lagran_init"] else 0))
        self.jt_total = rp["jt_total"]
        self.jt = 0
        return rp

    def state_dict(self, names=None) -> dict:
        names = capi.FIELDS if names is None else names
        d = {n: self.download(n) for n in names}
        for pn in capi.PLANES:
            d[pn] = self.download_plane(pn)
        return d
