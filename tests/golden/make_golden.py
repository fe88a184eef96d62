"""Record the golden fixtures of the oracle (run: python tests/golden/make_golden.py).

The reference publishes no golden data and cannot be built here (Fortran +
MPI + FFTW + 2DECOMP&FFT are absent), so these fixtures are regression pins
of the oracle itself: small grids, a few steps, the fields a user looks at.
The GPU parity tests compare the CUDA library with the same oracle runs.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from oracle import les_oracle as O  # noqa: E402

CASES = {
    "lasd_padd_16x16x8_12steps": dict(params=dict(nx=16, ny=16, nz=8), steps=12, seed=1),
    "cstsmag_trunc_16x16x8_4steps": dict(params=dict(nx=16, ny=16, nz=8, dealias="trunc", sgs_model="cst_Smag"),
                                         steps=4, seed=2),
    "lasd_periodic_halo_32x16x8_11steps": dict(params=dict(nx=32, ny=16, nz=8, lag_halo="periodic"), steps=11,
                                               seed=3),
}
SAVED = ("u", "v", "w", "p", "rhsx", "rhsz", "txz", "cs_opt2", "F_LM", "F_MM")


def run_case(case: dict) -> dict:
    p = O.Params(**case["params"])
    ops = O.Ops(p)
    st = O.make_state(p, seed=case["seed"])
    diags = []
    for _ in range(case["steps"]):
        diags.append(O.les_step(ops, st))
    out = {n: getattr(st, n).copy() for n in SAVED}
    out["diagnostics"] = np.array(diags)
    out["u_star_avg"] = st.u_star_avg.copy()
    return out


def main():
    here = Path(__file__).resolve().parent
    for name, case in CASES.items():
        out = run_case(case)
        np.savez_compressed(here / f"{name}.npz", **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
