"""CPU checks of the C-ABI library and the host-side mirror (no GPU calls)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "lesgpu.h"


def _declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(les_\w+)\s*\(", text, re.M)))


@pytest.fixture(scope="module")
def lib():
    from new_repo_b200 import capi

    if not capi.LIB_PATH.exists():
        from new_repo_b200.build import build

        build()
    return capi.load()


def test_header_declares_entry_points():
    syms = _declared_symbols()
    for name in ("les_create", "les_step", "les_press_stag_array", "les_compute_dealias_convec",
                 "les_sgs_stress", "les_grad_velocity_filt", "les_div_stress", "les_wallstress"):
        assert name in syms


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in _declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_prototypes_cover_header(lib):
    from new_repo_b200 import capi

    declared = set(_declared_symbols()) - {"les_last_error", "les_noalloc_last_error"}  # return strings
    assert declared <= set(capi.PROTOTYPES), declared - set(capi.PROTOTYPES)


def test_null_arguments_return_invalid(lib):
    from new_repo_b200 import capi

    assert lib.les_create(None, None) == capi.LES_ERR_INVALID
    assert lib.les_step(None, 1, 1) == capi.LES_ERR_INVALID
    assert b"null" in lib.les_last_error()
    assert lib.les_destroy(None) == capi.LES_OK
    # the host-state step and the page-locking helpers check before any CUDA call
    assert lib.les_step_host(None, 1, 1, None, None, None, None) == capi.LES_ERR_INVALID
    assert lib.les_host_register(None, 8) == capi.LES_ERR_INVALID
    assert lib.les_host_unregister(None) == capi.LES_ERR_INVALID
    assert lib.les_set_wall_model(None, 0) == capi.LES_ERR_INVALID


def test_invalid_model_is_rejected_before_device_use(lib):
    from new_repo_b200 import LesError, RunParams

    with pytest.raises(LesError) as e:
        RunParams(sgs_model="smagorinsky_typo").to_c()
    assert e.value.code == 1


def test_field_ids_match_header():
    from new_repo_b200 import capi

    text = HEADER.read_text()
    body = text[text.index("typedef enum les_field"):text.index("} les_field;")]
    names = re.findall(r"LES_([A-Z_0-9]+)", body)
    names = [n for n in names if n != "NFIELDS"]
    assert [n.lower() for n in names] == [f.lower() for f in capi.FIELDS]


def test_namelist_mirror(tmp_path):
    """parameters_IO.f90:238-277 arithmetic on a reference-style namelist."""
    from new_repo_b200 import read_namelist

    nml = tmp_path / "parameters.nlst"
    nml.write_text("""&simulation_param
p_on_y = 1
p_on_z = 1
nx = 64
ny = 32
nz = 16
nt = 100
dt = 2d-4
dim_dt_flag = .false.
/
&physical_param
XY_pi = .true.
lx = 2.0d0
ly = 2.0d0
lz = 1.0d0
zi = 1.0d0
lbc_dz0 = 1.0d-4
pfx = 1.0d0
/
&sgs_param
Cs0 = 0.16d0
sgs_model = 'dyn_LagScaleDep'
cs_count = 5
dyn_init = 5
/
&momentum_bc
lbc_special = 'wall_law'
wall_model = 'wall_filter'
/
""")
    p, raw = read_namelist(nml)
    assert (p.nx, p.ny, p.nz) == (64, 32, 16)
    assert p.lx == pytest.approx(2 * 3.141592653589793)
    assert p.dx == p.lx / 64.0 and p.dz == 1.0 / 16.0
    assert p.z0 == 1e-4 and p.dt_nd == 2e-4
    assert p.sgs_model == "dyn_LagScaleDep" and p.lbc_special == "wall_law"


def test_missing_namelist_is_io_error(tmp_path):
    from new_repo_b200 import LesError, read_namelist

    with pytest.raises(LesError) as e:
        read_namelist(tmp_path / "nope.nlst")
    assert e.value.code == 22
