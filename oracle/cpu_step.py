"""ctypes binding of the compiled FP64 oracle (oracle/cpu_step.cpp) -- TEST AND
BASELINE INFRASTRUCTURE ONLY (tests/, bench.py's CPU legs; never the product).

`build()` compiles ``cpu_step.cpp`` with g++ and OpenMP into
``oracle/_lib/libcpustep.so``; `CpuStep` holds one state, mirrors a numpy
oracle state into it and advances it by `les_step` on every host core.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "cpu_step.cpp"
LIB = HERE / "_lib" / "libcpustep.so"
FLAGS = ["-O3", "-march=x86-64-v3", "-std=c++17", "-fcx-limited-range", "-fopenmp", "-fPIC", "-shared"]

FIELDS = ("u", "v", "w", "dudx", "dudy", "dudz", "dvdx", "dvdy", "dvdz", "dwdx", "dwdy", "dwdz",
          "p", "dpdx", "dpdy", "dpdz", "rhsx", "rhsy", "rhsz", "rhsx_f", "rhsy_f", "rhsz_f",
          "txx", "txy", "txz", "tyy", "tyz", "tzz", "cs_opt2", "nu_t",
          "F_LM", "F_MM", "F_QN", "F_NN", "beta", "u_lag", "v_lag", "w_lag")
PLANES = ("lbc_u", "lbc_v", "lbc_w", "ubc_u", "ubc_v", "ubc_w", "bottom_wk_press", "top_wk_press",
          "lbc_z0", "u_star_avg")
BC = {"drc": 1, "neu": 2}
SGS = {"cst_Smag": 0, "dyn_LagScaleDep": 2}
WALL = {"wall_filter": 0, "wall_inst": 1, "wall_homog": 2}

_lib = None


def build(force: bool = False) -> Path:
    """Compile the oracle's C++ restatement (g++ -fopenmp) if it is missing or
    older than its source."""
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        LIB.parent.mkdir(exist_ok=True)
        tmp = LIB.with_name(LIB.name + f".{os.getpid()}.tmp")
        r = subprocess.run(["g++", *FLAGS, "-o", str(tmp), str(SRC)], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"g++ failed for {SRC.name}:\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        lib = C.CDLL(str(build()))
        d, i, vp, dp, ip = C.c_double, C.c_int, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        lib.cs_create.restype = vp
        lib.cs_create.argtypes = [i, i, i, d, d, d, d, d, d, d, d, i, i, i, i]
        lib.cs_destroy.argtypes = [vp]
        for f in (lib.cs_set_field, lib.cs_get_field, lib.cs_set_plane, lib.cs_get_plane):
            f.argtypes = [vp, i, dp]
        lib.cs_set_flags.argtypes = [vp, i, i, i, ip, ip]
        lib.cs_set_threads.argtypes = [i]
        lib.cs_max_threads.restype = i
        lib.cs_step.argtypes = [vp, i, dp]
        lib.cs_step.restype = i
        lib.cs_rfft2.argtypes = [i, i, dp, dp]
        lib.cs_irfft2.argtypes = [i, i, dp, dp]
        _lib = lib
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def rfft2(f: np.ndarray) -> np.ndarray:
    """Unnormalised 2-D r2c of one (ny, nx) plane."""
    ny, nx = f.shape
    f = np.ascontiguousarray(f, dtype=np.float64)
    out = np.zeros((ny, nx // 2 + 1), dtype=np.complex128)
    load().cs_rfft2(nx, ny, _ptr(f), out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def irfft2(F: np.ndarray, nx: int) -> np.ndarray:
    """Unnormalised 2-D c2r to an (ny, nx) plane."""
    ny = F.shape[0]
    F = np.array(F, dtype=np.complex128, order="C")
    out = np.zeros((ny, nx))
    load().cs_irfft2(nx, ny, F.ctypes.data_as(C.POINTER(C.c_double)), _ptr(out))
    return out


class CpuStep:
    """One compiled-oracle state with the parameters of an oracle Params."""

    def __init__(self, p, threads: int | None = None):
        lib = load()
        if threads is not None:
            lib.cs_set_threads(int(threads))
        self.p = p
        self.h = lib.cs_create(p.nx, p.ny, p.nz, p.dt, p.lx, p.ly, p.lz, p.z0, p.pfx, p.pfy, p.cs0,
                               SGS[p.sgs_model], p.cs_count, p.dyn_init, WALL[p.wall_model])
        if not self.h:
            raise ValueError("cpu_step: unsupported configuration")
        if p.lbc_special != "wall_law" or p.dealias != "padd" or p.lag_halo != "reference1x1":
            raise ValueError("cpu_step covers the wall law, 3/2 padding and the reference1x1 halos")

    def close(self):
        if self.h:
            load().cs_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def mirror(self, st) -> None:
        """Copy every field, plane and flag of a numpy oracle State."""
        lib = load()
        for q, n in enumerate(FIELDS):
            a = np.ascontiguousarray(getattr(st, n), dtype=np.float64)
            lib.cs_set_field(self.h, q, _ptr(a))
        for q, n in enumerate(PLANES):
            a = np.ascontiguousarray(getattr(st, n), dtype=np.float64)
            lib.cs_set_plane(self.h, q, _ptr(a))
        lbc = (C.c_int * 3)(*[BC[st.lbc_typ[c]] for c in "uvw"])
        ubc = (C.c_int * 3)(*[BC[st.ubc_typ[c]] for c in "uvw"])
        lib.cs_set_flags(self.h, int(st.f_coeff_init), int(st.lagran_init), int(st.jt_total), lbc, ubc)

    def step(self, n: int = 1):
        d = np.zeros(4)
        if load().cs_step(self.h, int(n), _ptr(d)) != 0:
            raise RuntimeError("cpu_step: step failed")
        return tuple(d)

    def field(self, name: str) -> np.ndarray:
        p = self.p
        out = np.zeros((p.nz + 2, p.ny, p.nx))
        load().cs_get_field(self.h, FIELDS.index(name), _ptr(out))
        return out

    def plane(self, name: str) -> np.ndarray:
        out = np.zeros((self.p.ny, self.p.nx))
        load().cs_get_plane(self.h, PLANES.index(name), _ptr(out))
        return out
