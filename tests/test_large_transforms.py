"""Parity of the spectral operators at the transform lengths of production
grids, against the FP64 oracle on a few levels.

The per-operator tests use 32- and 64-point grids; here nx = ny = 256 and 512
reach the three-pass register FFTs (384, 512 and 768 points: the x and y
transforms of the 3/2-padded convective term) and the 256-point plans of the
256^3 bench, with the exchange layouts and twiddle tables chosen per plan.
Tolerances as elsewhere: 1e-12 (FP64), 1e-5 (mixed, on FP32-rounded
inputs)."""
import numpy as np
import pytest

from oracle import les_oracle as O
from tests.helpers import mirror, rel_err, run_params

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "mixed": 1e-5}


def _setup(n, precision, dealias="padd", nz=2, seed=4):
    from new_repo_b200 import LES

    p = O.Params(nx=n, ny=n, nz=nz, dealias=dealias)
    ops = O.Ops(p)
    st = O.make_state(p, seed=seed)
    O.compute_vel_grad(ops, st)
    if precision == "mixed":
        for name in O.FIELDS:
            a = getattr(st, name)
            a[...] = a.astype(np.float32).astype(np.float64)
    les = LES(run_params(p), precision=precision)
    mirror(les, st)
    return p, ops, st, les


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n", [256, 512])
def test_grad_velocity_filt_large(gpu, n, precision):
    p, ops, st, les = _setup(n, precision)
    O.grad_velocity_filt(ops, st.u, st.dudx, st.dudy)
    les.grad_velocity_filt("u", "dudx", "dudy")
    for name in ("u", "dudx", "dudy"):
        e = rel_err(les.download(name), getattr(st, name))
        assert e <= TOL[precision], (n, precision, name, e)
    les.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n,dealias", [(256, "padd"), (512, "padd"), (256, "trunc")])
def test_dealias_convec_large(gpu, n, dealias, precision):
    p, ops, st, les = _setup(n, precision, dealias)
    O.compute_dealias_convec(p, st, st.rhsx, st.rhsy, st.rhsz)
    les.compute_dealias_convec("rhsx", "rhsy", "rhsz")
    for name in ("rhsx", "rhsy", "rhsz"):
        e = rel_err(les.download(name), getattr(st, name))
        assert e <= TOL[precision], (n, dealias, precision, name, e)
    les.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_press_stag_array_large(gpu, precision):
    p, ops, st, les = _setup(256, precision, nz=4)
    O.press_stag_array(ops, st, 1.0)
    les.press_stag_array(1.0)
    for name in ("p", "dpdx", "dpdy", "dpdz"):
        e = rel_err(les.download(name), getattr(st, name))
        assert e <= TOL[precision], (precision, name, e)
    les.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nx,ny", [(16, 128), (128, 16)])
def test_small_and_asymmetric_plans(gpu, nx, ny, precision):
    """Single-pass plans (8-24 points: one lane per sequence, many sequences
    per warp) against multi-pass ones in the other direction."""
    from new_repo_b200 import LES

    p = O.Params(nx=nx, ny=ny, nz=4)
    ops = O.Ops(p)
    st = O.make_state(p, seed=5)
    O.compute_vel_grad(ops, st)
    if precision == "mixed":
        for name in O.FIELDS:
            a = getattr(st, name)
            a[...] = a.astype(np.float32).astype(np.float64)
    les = LES(run_params(p), precision=precision)
    mirror(les, st)
    O.grad_velocity_filt(ops, st.v, st.dvdx, st.dvdy)
    les.grad_velocity_filt("v", "dvdx", "dvdy")
    O.compute_dealias_convec(p, st, st.rhsx, st.rhsy, st.rhsz)
    les.compute_dealias_convec("rhsx", "rhsy", "rhsz")
    for name in ("v", "dvdx", "dvdy", "rhsx", "rhsy", "rhsz"):
        e = rel_err(les.download(name), getattr(st, name))
        assert e <= TOL[precision], (nx, ny, precision, name, e)
    les.close()
