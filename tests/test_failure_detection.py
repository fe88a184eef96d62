"""Failure detection and recovery, with the failures made on the host.

The reference aborts with decomp_2d_abort code 9 when check_NaN finds a NaN
in u, v, w (LES_engine.f90:583-616, every NaN_check = 20 steps) and when the
tridiagonal elimination meets a zero pivot (compute_pressure.f90:411-418).
Here the device sets sticky status bits (ST_NAN in the diagnostics kernel,
ST_PIVOT in the tridiagonal kernel) and les_check_status turns them into
status 9 with the reference's message, leaving the state usable so that a
driver can reload its last checkpoint and go on.

Nothing here faults the GPU: the NaN is planted in a host array before it is
uploaded, and the singular system comes from a host-built grid whose
wavenumbers underflow to zero (every (kx, ky) column then has the Neumann-
Neumann matrix of the mean mode, whose last pivot is exactly zero).
"""
import numpy as np
import pytest

from new_repo_b200.capi import LES_ERR_INVALID, LES_ERR_NUMERICAL, LesError


def _params(**kw):
    from new_repo_b200 import RunParams

    base = dict(nx=32, ny=32, nz=16, dt=2e-4, sgs_model="dyn_LagScaleDep", nan_check=1)
    base.update(kw)
    return RunParams(**base)


def test_status_codes_are_distinct():
    from new_repo_b200 import capi

    codes = [capi.LES_ERR_INVALID, capi.LES_ERR_NOMEM, capi.LES_ERR_DEVICE, capi.LES_ERR_NUMERICAL, capi.LES_ERR_IO]
    assert len(set(codes)) == len(codes)
    assert (capi.LES_ERR_NOMEM, capi.LES_ERR_NUMERICAL) == (3, 9)


def test_check_status_needs_a_state():
    from new_repo_b200 import capi

    lib = capi.load()
    assert lib.les_check_status(None, None) == LES_ERR_INVALID


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nan_in_uploaded_velocity_gives_status_9(gpu, precision):
    from oracle import les_oracle as O
    from new_repo_b200 import LES

    p = _params()
    les = LES(p, precision=precision)
    u, v, w = O.log_law_fields(O.Params(nx=p.nx, ny=p.ny, nz=p.nz), seed=1)
    les.set_initial_conditions(u, v, w)
    les.step(2)
    assert les.check_status() == 0
    bad = les.download("v")
    bad[5, 3, 7] = np.nan
    les.upload("v", bad)
    with pytest.raises(LesError) as e:
        les.step(1)  # nan_check = 1: check_NaN after every step
    assert e.value.code == LES_ERR_NUMERICAL
    assert "NaN" in str(e.value)
    # the bits were read and cleared: the state answers again
    assert les.check_status() == 0
    les.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_zero_pivot_gives_status_9(gpu, precision):
    """Domain lengths of 1e200: 2 pi / lx squared underflows, every column's
    system is singular and the top-row pivot is 0 (bet = 1 - 1)."""
    from new_repo_b200 import LES, capi

    p = _params(xy_pi=False, lx_in=1e200, ly_in=1e200, sgs_model="cst_Smag")
    les = LES(p, precision=precision)
    rng = np.random.default_rng(2)
    shp = (p.nz + 2, p.ny, p.nx)
    for f in ("u", "v", "w"):
        les.upload(f, rng.standard_normal(shp))
    les.press_stag_array(1.0)
    with pytest.raises(LesError) as e:
        les.check_status()
    assert e.value.code == LES_ERR_NUMERICAL
    assert "bet(i,j)=0" in str(e.value)
    # a regular grid in the same process is unaffected
    q = LES(_params(sgs_model="cst_Smag"), precision=precision)
    for f in ("u", "v", "w"):
        q.upload(f, rng.standard_normal(shp))
    q.press_stag_array(1.0)
    assert q.check_status() == 0
    q.close()
    les.close()


@pytest.mark.gpu
def test_recovery_from_checkpoint_after_nan(gpu, tmp_path):
    """status 9 -> reload the last checkpoint -> continue: the recovered run
    equals a run that restarted from the same checkpoint without the NaN,
    bit for bit."""
    from oracle import les_oracle as O
    from new_repo_b200 import LES

    p = _params(dyn_init=2, cs_count=2)
    a = LES(p)
    a.set_initial_conditions(*O.log_law_fields(O.Params(nx=p.nx, ny=p.ny, nz=p.nz), seed=3))
    a.step(4)
    a.checkpoint_out(tmp_path)
    # clean continuation from the checkpoint
    ref = LES(p)
    ref.checkpoint_in(tmp_path)
    ref.step(3)
    # failing run: NaN after the checkpoint, detected, reloaded, continued
    a.step(1)
    u = a.download("u")
    u[3, 4, 5] = np.nan
    a.upload("u", u)
    with pytest.raises(LesError) as e:
        a.step(1)
    assert e.value.code == LES_ERR_NUMERICAL
    a.checkpoint_in(tmp_path)
    a.step(3)
    for n in ("u", "v", "w", "p", "cs_opt2", "rhsx", "txz", "F_LM"):
        x, y = a.download(n)[1:-1], ref.download(n)[1:-1]
        assert np.array_equal(x, y), n
    assert a.jt_total == ref.jt_total
    a.close()
    ref.close()
