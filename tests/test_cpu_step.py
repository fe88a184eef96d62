"""The compiled FP64 oracle (oracle/cpu_step.cpp, the CPU baseline of bench.py)
against the numpy oracle it restates.

Its transforms match scipy's to rounding; its time steps follow the numpy
oracle's through LASD updates (the F-initialising update and the Lagrangian
interpolation of later ones).  Tolerances (normwise relative per field after
the stated steps): u, v, w, p and their gradients <= 1e-10; the SGS fields
and the right-hand sides <= 5e-7, because the reference's REAL(4) roundings
of cs_opt2, beta, F_LM and F_QN can land on the neighbouring float when two
FP64 computations differ in the last bit, and that moves those points by a
float ulp; diagnostics cfl, mke, u* to 1e-12 (rms div u is a rounding-level
quantity and is not compared).
"""
import numpy as np
import pytest
import scipy.fft as sfft

from oracle import cpu_step as CS
from oracle import les_oracle as O

SGS_RHS = {"cs_opt2", "beta", "F_LM", "F_QN", "F_MM", "F_NN", "nu_t", "txx", "txy", "txz", "tyy", "tyz", "tzz",
           "rhsx", "rhsy", "rhsz", "rhsx_f", "rhsy_f", "rhsz_f"}


@pytest.mark.parametrize("ny,nx", [(16, 16), (32, 24), (48, 96), (256, 384)])
def test_transforms_match_scipy(ny, nx):
    rng = np.random.default_rng(ny * 1000 + nx)
    f = rng.standard_normal((ny, nx))
    F = CS.rfft2(f)
    R = sfft.rfft2(f)
    assert np.abs(F - R).max() <= 2e-15 * np.abs(R).max()
    g = CS.irfft2(R, nx)
    G = sfft.irfft2(R, s=(ny, nx), norm="forward")
    assert np.abs(g - G).max() <= 2e-15 * np.abs(G).max()


@pytest.mark.parametrize("cfg,steps", [
    (dict(nx=32, ny=32, nz=16), 10),
    (dict(nx=48, ny=32, nz=8, dyn_init=1, cs_count=2), 6),
    (dict(nx=32, ny=48, nz=8, sgs_model="cst_Smag", wall_model="wall_inst"), 4),
])
def test_steps_follow_the_numpy_oracle(cfg, steps):
    p = O.Params(**cfg)
    ops = O.Ops(p)
    st = O.make_state(p, seed=1)
    cs = CS.CpuStep(p, threads=4)
    cs.mirror(st)
    for n in range(steps):
        d_o = O.les_step(ops, st)
        d_c = cs.step()
        assert np.allclose(d_c[:3], d_o[:3], rtol=1e-12, atol=1e-15), (n, d_c, d_o)
    for name in CS.FIELDS:
        a = cs.field(name)[1:p.nz + 1]
        b = getattr(st, name)[1:p.nz + 1]
        den = np.abs(b).max()
        e = float(np.abs(a - b).max() / den) if den > 0 else float(np.abs(a - b).max())
        assert e <= (5e-7 if name in SGS_RHS else 1e-10), (name, e)
    for name in ("u_star_avg", "lbc_u", "bottom_wk_press"):
        a, b = cs.plane(name), getattr(st, name)
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(b).max(), 1e-300), name
    cs.close()
