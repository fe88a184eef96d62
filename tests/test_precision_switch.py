"""les_set_precision: a state moves between FP64 and mixed precision with its
fields, planes, boundary-condition types and Lagrangian flags."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _les(precision):
    from new_repo_b200 import LES, RunParams, log_law_noise

    p = RunParams(nx=32, ny=32, nz=16, dt=2e-4, sgs_model="dyn_LagScaleDep", dyn_init=2, cs_count=2)
    les = LES(p, precision=precision)
    les.set_initial_conditions(*log_law_noise(p, seed=3))
    return les


def test_switch_carries_the_state(gpu):
    ref = _les("fp64")
    sw = _les("fp64")
    ref.step(4)
    sw.step(4)
    names = ("u", "v", "w", "cs_opt2", "F_LM", "F_MM", "rhsx")
    before = {n: sw.download(n) for n in names}
    planes = {n: sw.download_plane(n) for n in ("lbc_u", "u_star_avg")}
    flag = sw.f_coeff_init
    sw.set_precision("mixed")
    assert sw.precision == "mixed" and sw.f_coeff_init == flag
    for n in names:  # FP32 fields: round to nearest
        np.testing.assert_array_equal(sw.download(n), before[n].astype(np.float32).astype(np.float64), err_msg=n)
    for n, a in planes.items():
        np.testing.assert_array_equal(sw.download_plane(n), a.astype(np.float32).astype(np.float64), err_msg=n)
    # the run continues in mixed precision close to the FP64 run
    ref.step(3)
    sw.step(3)
    for n in ("u", "v", "w"):
        a, b = sw.download(n)[1:-1], ref.download(n)[1:-1]
        assert np.abs(a - b).max() <= 1e-4 * np.abs(b).max(), n
    # and back: FP64 holds the FP32 values exactly
    mid = sw.download("u")
    sw.set_precision("fp64")
    np.testing.assert_array_equal(sw.download("u"), mid)
    sw.step(1)
    ref.close()
    sw.close()


def test_switch_refused_with_the_learned_closure(gpu):
    from new_repo_b200 import LesError

    les = _les("fp64")
    les.set_sgs_model("mlp")
    with pytest.raises(LesError) as e:
        les.set_precision("mixed")
    assert e.value.code == 1
    with pytest.raises(LesError):
        les.set_precision("fp16")
    les.close()
