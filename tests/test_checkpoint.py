"""Checkpoint / restart: the file of IO_checkpoint.f90:119-256 (one rank) and
the restart namelist of parameters_IO.f90:333-435.

The GPU writes the same bytes as the oracle's restatement of the format,
reads the oracle's files back exactly, and a run restarted from a checkpoint
continues like the uninterrupted run (FP64: within 1e-12 relative)."""
import numpy as np
import pytest

from oracle import les_oracle as O
from tests.helpers import mirror, oracle_run, run_params


def test_oracle_checkpoint_round_trip(tmp_path):
    p = O.Params(nx=16, ny=16, nz=8, dyn_init=5, cs_count=5)
    _, st = oracle_run(p, 10)  # step 10 is a dynamic update: the F averages exist
    assert st.lagran_init
    path = tmp_path / "checkpoint_000000010"
    O.write_checkpoint(st, path)
    assert path.stat().st_size == 11 * 16 * 16 * 9 * 8
    back = O.State(p)
    O.read_checkpoint(back, path, True)
    for n in O.CHECKPOINT_FIELDS + O.CHECKPOINT_F:
        np.testing.assert_array_equal(getattr(back, n)[1:], getattr(st, n)[1:])
    assert back.f_coeff_init and back.lagran_init


def test_checkpoint_follows_the_reference_reader(tmp_path):
    """The reference's reader (matlab_src/load2decomp_checkpoint.m), restated:
    u v w RHSx RHSy RHSz Cs_opt2 [F_LM F_MM F_QN F_NN], each nx*ny*(nz+1)
    doubles in Fortran order (levels 1..nz+1)."""
    p = O.Params(nx=16, ny=8, nz=4, dyn_init=5, cs_count=5)
    _, st = oracle_run(p, 10)
    path = tmp_path / "checkpoint_000000010"
    O.write_checkpoint(st, path)
    raw = np.fromfile(path, dtype="<f8")
    n = p.nx * p.ny * (p.nz + 1)
    names = ("u", "v", "w", "rhsx", "rhsy", "rhsz", "cs_opt2", "F_LM", "F_MM", "F_QN", "F_NN")
    assert raw.size == len(names) * n
    for q, name in enumerate(names):
        arr = raw[q * n:(q + 1) * n].reshape((p.nx, p.ny, p.nz + 1), order="F")
        np.testing.assert_array_equal(arr, getattr(st, name)[1:].transpose(2, 1, 0), err_msg=name)


def test_restart_namelist_round_trip(tmp_path):
    from new_repo_b200 import LesError, RunParams
    from new_repo_b200.les import read_parameters_restart, write_parameters_restart

    p = RunParams(nx=32, ny=16, nz=8, dt=1e-4, sgs_model="dyn_LagScaleDep", dyn_init=5)
    f = tmp_path / "parameters_restart.nlst"
    write_parameters_restart(f, p, 1234, True)
    rp = read_parameters_restart(f, p)
    assert rp == {"jt_total": 1234, "dyn_init": 5, "lagran_init": True, "sgs_model": "dyn_LagScaleDep"}
    with pytest.raises(LesError) as e:
        read_parameters_restart(f, RunParams(nx=64, ny=16, nz=8))
    assert e.value.code == 1
    with pytest.raises(LesError) as e:
        read_parameters_restart(tmp_path / "missing.nlst", p)
    assert e.value.code == 22


def _les(p):
    from new_repo_b200 import LES

    return LES(run_params(p), precision="fp64")


@pytest.mark.gpu
def test_checkpoint_bytes_match_the_reference_format(gpu, tmp_path):
    p = O.Params(nx=32, ny=16, nz=8, dyn_init=5, cs_count=5)
    _, st = oracle_run(p, 10)
    les = _les(p)
    mirror(les, st)
    les.jt_total = 10
    # lagran_init is the solver's flag; mirror() set it through f_coeff_init
    path = les.checkpoint_out(tmp_path)
    ref = tmp_path / "oracle_checkpoint"
    O.write_checkpoint(st, ref)
    assert path.read_bytes() == ref.read_bytes()
    les.close()


@pytest.mark.gpu
def test_checkpoint_read_restores_fields(gpu, tmp_path):
    p = O.Params(nx=32, ny=16, nz=8, dyn_init=5, cs_count=5)
    _, st = oracle_run(p, 10)
    O.write_checkpoint(st, tmp_path / "checkpoint_000000010")
    from new_repo_b200.les import write_parameters_restart

    les = _les(p)
    write_parameters_restart(tmp_path / "parameters_restart.nlst", les.params, 10, True)
    rp = les.checkpoint_in(tmp_path)
    assert rp["jt_total"] == 10 and les.jt_total == 10 and les.f_coeff_init
    for n in O.CHECKPOINT_FIELDS + O.CHECKPOINT_F:
        np.testing.assert_array_equal(les.download(n)[1:], getattr(st, n)[1:])
    les.close()


@pytest.mark.gpu
def test_restart_continues_the_run(gpu, tmp_path):
    p = O.Params(nx=32, ny=32, nz=16, dyn_init=5, cs_count=5)
    from new_repo_b200 import log_law_noise

    a = _les(p)
    a.set_initial_conditions(*log_law_noise(a.params, seed=2))
    a.step(10)  # a dynamic update at step 10 empties the Lagrangian accumulators
    a.checkpoint_out(tmp_path)
    b = _les(p)
    b.checkpoint_in(tmp_path)
    a.step(7)
    b.step(7)
    for n in ("u", "v", "w", "cs_opt2", "F_LM", "F_MM", "p"):
        x, y = a.download(n)[1:p.nz + 1], b.download(n)[1:p.nz + 1]
        err = np.abs(x - y).max() / max(np.abs(x).max(), 1e-300)
        assert err <= 1e-12, (n, err)
    a.close()
    b.close()
