"""ctypes binding of liblesgpu.so (the C ABI declared in include/lesgpu.h).

The shared library is built in-tree by ``new_repo_b200/build.py``.  Loading
fails loudly when it is missing: there is no CPU fallback for any operator.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "liblesgpu.so"

LES_OK, LES_ERR_INVALID, LES_ERR_NOMEM, LES_ERR_DEVICE, LES_ERR_NUMERICAL, LES_ERR_IO = 0, 1, 3, 4, 9, 22
SGS_MODELS = {"cst_Smag": 0, "dyn_Smag": 1, "dyn_LagScaleDep": 2, "mlp": 3}
MLP_NPARAM = 4801
MLP_NSTATS = 36
WALL_MODELS = {"wall_filter": 0, "wall_inst": 1, "wall_homog": 2}
DEALIAS = {"padd": 0, "trunc": 1}
LAG_HALO = {"reference1x1": 0, "periodic": 1}
PRECISION = {"fp64": 0, "mixed": 1}

FIELDS = ("u", "v", "w", "dudx", "dudy", "dudz", "dvdx", "dvdy", "dvdz", "dwdx", "dwdy", "dwdz",
          "p", "dpdx", "dpdy", "dpdz", "rhsx", "rhsy", "rhsz", "rhsx_f", "rhsy_f", "rhsz_f",
          "txx", "txy", "txz", "tyy", "tyz", "tzz", "cs_opt2", "nu_t",
          "F_LM", "F_MM", "F_QN", "F_NN", "beta", "u_lag", "v_lag", "w_lag",
          "theta", "dtdx", "dtdy", "dtdz", "rhs_t", "rhs_t_f", "qx", "qy", "qz")
SCALAR_SGS = {"const": 0, "dynamic": 1}
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}
PLANES = ("lbc_u", "lbc_v", "lbc_w", "ubc_u", "ubc_v", "ubc_w", "bottom_wk_press", "top_wk_press",
          "lbc_z0", "u_star_avg")
PLANE_ID = {n: i for i, n in enumerate(PLANES)}


class LesParams(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dt", C.c_double),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double), ("z0", C.c_double),
                ("pfx", C.c_double), ("pfy", C.c_double), ("cs0", C.c_double),
                ("sgs_model", C.c_int), ("cs_count", C.c_int), ("dyn_init", C.c_int),
                ("wall_law", C.c_int), ("wall_model", C.c_int), ("dealias", C.c_int),
                ("lag_halo", C.c_int), ("precision", C.c_int), ("device", C.c_int)]


class ScalarParams(C.Structure):
    _fields_ = [("surface_flux", C.c_double), ("top_gradient", C.c_double), ("buoyancy", C.c_double),
                ("pr_t", C.c_double), ("sgs", C.c_int)]


class LesError(RuntimeError):
    """A nonzero status from the library; ``code`` mirrors decomp_2d_abort codes."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


# (name, argtypes) of every exported entry point
_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.c_int
_F = C.POINTER(C.c_float)
PROTOTYPES = {
    "les_create": [C.POINTER(LesParams), C.POINTER(_P)],
    "les_destroy": [_P],
    "les_upload": [_P, _I, _D, _I, _I],
    "les_download": [_P, _I, _D, _I, _I],
    "les_upload_plane": [_P, _I, _D],
    "les_download_plane": [_P, _I, _D],
    "les_set_initial_conditions": [_P, _D, _D, _D],
    "les_set_bc_types": [_P, C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "les_set_lagrangian_init": [_P, _I],
    "les_get_lagrangian_init": [_P, C.POINTER(C.c_int)],
    "les_grad_velocity_filt": [_P, _I, _I, _I],
    "les_ddz_uv": [_P, _I, _I],
    "les_ddz_w": [_P, _I, _I],
    "les_div_stress": [_P, _I, _I, _I, _I, _I],
    "les_compute_dealias_convec": [_P, _I, _I, _I],
    "les_press_stag_array": [_P, C.c_double],
    "les_press_from_increment": [_P, C.c_double, C.c_double],
    "les_set_pressure_slabs": [_P, _I],
    "les_obukhov": [_P],
    "les_wallstress": [_P],
    "les_sgs_stress": [_P, _I, _I],
    "les_test_filter": [_P, _I, _I],
    "les_set_bc": [_P],
    "les_compute_vel_grad": [_P],
    "les_compute_rhs_adv": [_P],
    "les_ab2_advance": [_P, C.c_double, C.c_double],
    "les_projection": [_P, C.c_double],
    "les_step": [_P, _I, _I],
    "les_diagnostics": [_P, _D],
    "les_get_status": [_P, C.POINTER(C.c_uint)],
    "les_check_status": [_P, C.POINTER(C.c_uint)],
    "les_scalar_init": [_P, C.POINTER(ScalarParams)],
    "les_scalar_set_initial": [_P, _D],
    "les_scalar_kappa": [_P, _D, _I],
    "les_sponge_init": [_P, C.c_double],
    "les_set_coriolis": [_P, C.c_double, C.c_double, C.c_double],
    "les_set_cs2_max": [_P, C.c_double],
    "les_sync": [_P],
    "les_timers": [_P, _D],
    "les_profile": [_P, _I],
    "les_profile_report": [_P, C.c_char_p, _I],
    "les_launch_count": [_P, C.POINTER(C.c_longlong)],
    "les_event_record": [_P, _I],
    "les_event_elapsed": [_P, _I, _I, _D],
    "les_upload_async": [_P, _I, C.c_void_p, _I, _I],
    "les_download_async": [_P, _I, C.c_void_p, _I, _I],
    "les_diagnostics_async": [_P, C.c_void_p],
    "les_set_wall_model": [_P, _I],
    "les_step_host": [_P, _I, _I, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "les_host_register": [C.c_void_p, C.c_size_t],
    "les_host_unregister": [C.c_void_p],
    "les_checkpoint_write": [_P, C.c_char_p],
    "les_checkpoint_read": [_P, C.c_char_p, _I],
    "les_set_precision": [_P, _I],
    "les_stat_init": [_P],
    "les_stat_averages": [_P, _I, _I, _I, _I, C.c_char_p],
    "les_stat_sums": [_P, _I, _D],
    "les_stat_iterations": [_P, C.POINTER(_I)],
    "les_stat_spectra": [_P, _I, _I, C.c_char_p],
    "les_tke_init": [_P, C.c_char_p],
    "les_tke_budget": [_P, _I, _I],
    "les_tke_sums": [_P, _D, C.POINTER(_I)],
    "les_set_sgs_model": [_P, _I],
    "les_mlp_init": [_P, C.c_uint],
    "les_mlp_set_params": [_P, _F, _I],
    "les_mlp_get_params": [_P, _F, _I],
    "les_mlp_reset_data": [_P, C.c_long],
    "les_mlp_collect": [_P, _I, _I, _I, C.c_uint],
    "les_mlp_counts": [_P, C.POINTER(C.c_longlong)],
    "les_mlp_fit_stats": [_P],
    "les_mlp_train": [_P, _I, _I, C.c_double, _D, _D],
    "les_mlp_forward": [_P, _F, C.c_long, _F],
    "les_mlp_grad": [_P, _F, _F, C.c_long, _F, _F],
    "les_mlp_info": [_P, _D],
    "les_mlp_set_check_every": [_P, _I],
    "les_mlp_set_wall_levels": [_P, _I],
    "les_mlp_check_profile": [_P, _D, _I],
    "les_grad_xy_noalloc": [_P, _P, _P, _I, _I, _I, C.c_double, C.c_double, _P],
}

_lib = None


# running sums of IO_statistics.f90:447-488, in the order of the RAV_*_3D.dat file
STAT_NAMES = ("u", "v", "w", "p", "u2", "v2", "w2", "u3", "v3", "w3", "u4", "v4", "w4", "uv", "uw", "vw",
              "txx", "tyy", "tzz", "txy", "txz", "tyz", "dudz", "dvdz", "nut", "cs")
# TKE budget profiles of tke_budget1D.f90:218-383, in the order of its avg_var calls
TKE_NAMES = ("u", "v", "w", "dudx", "dudy", "dudz", "dvdx", "dvdy", "dvdz", "dwdx", "dwdy", "dwdz",
             "uu", "vv", "ww", "uv", "uw", "vw", "txx", "tyy", "tzz", "txy", "txz", "tyz", "cs",
             "uuw", "vvw", "www", "uww", "wtzz", "utxz", "vtyz", "dxx", "dyy", "dzz", "dxy", "dxz", "dyz",
             "dudx2", "dudy2", "dudz2", "dvdx2", "dvdy2", "dvdz2", "dwdx2", "dwdy2", "dwdz2",
             "dudxdwdx", "dudydwdy", "dudzdwdz",
             "p", "dpdx", "dpdy", "dpdz", "pw", "pu", "pdudx", "pdvdy", "pdwdz", "pdwdx", "pdudz")


def load() -> C.CDLL:
    """Load liblesgpu.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run new_repo_b200/build.py (or __graft_entry__.build())")
        lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | getattr(os, "RTLD_GLOBAL", 0))
        for name, argt in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.argtypes = argt
            fn.restype = C.c_int
        lib.les_last_error.argtypes = []
        lib.les_last_error.restype = C.c_char_p
        lib.les_noalloc_last_error.argtypes = []
        lib.les_noalloc_last_error.restype = C.c_char_p
        _lib = lib
    return _lib


def check(rc: int) -> None:
    if rc != LES_OK:
        msg = load().les_last_error().decode(errors="replace")
        raise LesError(rc, msg)
