"""z-slab decomposition pieces: the partitioned tridiagonal solve (the
pressure systems solved where a z-slab rank holds them, instead of the
reference's transposes to columns, compute_pressure.f90:265,290) and the
ghost-plane exchange (update_ghost / update_halo3, decomp_2d_custom.f90:
324-473, 902-1024).

CPU: the partition method of oracle/slab_oracle.py against the single-sweep
Thomas solve of the oracle; the distributed host logic (new_repo_b200.slabs)
over gloo at world sizes 2 and 4 against the one-domain answers.  GPU: the
library's partitioned pressure solve (les_set_pressure_slabs) against the
single sweep, FP64 <= 1e-12 and mixed <= 1e-5 (the same bars as every
pressure test)."""
import os

import numpy as np
import pytest

from oracle import les_oracle as O
from oracle import slab_oracle as Z


def _system(p, seed=0):
    ops = O.Ops(p)
    a, b, c = O.tridiag_coeffs(ops)
    rng = np.random.default_rng(seed)
    r = rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape)
    return ops, a, b, c, r


@pytest.mark.parametrize("G", [1, 2, 4, 8])
def test_partitioned_solve_equals_thomas(G):
    p = O.Params(nx=16, ny=16, nz=64)
    ops, a, b, c, r = _system(p)
    x0 = O.tridiag_solver_parallel(ops, r)
    x = Z.partitioned_solve(a, b, c, r, G)
    x[:, :, p.lhx - 1] = 0.0
    x[:, p.lhy - 1, :] = 0.0
    err = np.abs(x - x0).max() / np.abs(x0).max()
    assert err <= 1e-12, (G, err)


def test_slab_rows_cover_the_column():
    rows = Z.slab_rows(64, 4)
    assert rows[0][0] == 0 and rows[-1][1] == 65
    assert all(rows[i][1] + 1 == rows[i + 1][0] for i in range(3))
    with pytest.raises(ValueError):
        Z.slab_rows(10, 4)


def _free_port() -> int:
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _slab_worker(rank, world, port, q):
    import sys

    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    from new_repo_b200 import slabs

    # the pressure systems of a 16 x 16 x 32 grid, the same on every rank
    p = O.Params(nx=16, ny=16, nz=32)
    ops, a, b, c, r = _system(p, seed=3)
    x0 = O.tridiag_solver_parallel(ops, r)
    s, e = slabs.slab_rows(p.nz, world, rank)
    t = lambda z: torch.from_numpy(np.ascontiguousarray(z[s:e + 1]))  # noqa: E731
    x = slabs.partitioned_solve(dist, t(a), t(b), t(c), t(r)).numpy()
    x[:, :, p.lhx - 1] = 0.0
    x[:, p.lhy - 1, :] = 0.0
    err_solve = float(np.abs(x - x0[s:e + 1]).max() / np.abs(x0).max())
    # ghost planes of a field's slab
    f = np.random.default_rng(5).standard_normal((p.nz + 2, p.ny, p.nx))
    m = p.nz // world
    loc = torch.zeros((m + 2, p.ny, p.nx), dtype=torch.float64)
    loc[1:m + 1] = torch.from_numpy(f[rank * m + 1:(rank + 1) * m + 1])
    if rank == 0:
        loc[0] = torch.from_numpy(f[0])
    if rank == world - 1:
        loc[m + 1] = torch.from_numpy(f[p.nz + 1])
    slabs.halo_exchange(dist, loc)
    below, above = Z.halo_planes(f, world)[rank]
    err_halo = float(max(np.abs(loc[0].numpy() - below).max(), np.abs(loc[m + 1].numpy() - above).max()))
    dist.barrier()
    q.put((rank, err_solve, err_halo))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_distributed_slabs_gloo(world):
    """Each rank holds its slab's rows; the distributed partitioned solve
    equals the one-domain Thomas solve to 1e-12, and the exchanged ghost
    planes equal the one-domain field's neighbouring levels exactly."""
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_worker, args=(r, world, port, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=180)
        assert pr.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, es, eh in res:
        assert es <= 1e-12, (rank, es)
        assert eh == 0.0, (rank, eh)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("G", [2, 4, 8])
def test_pressure_slabs_match_single_sweep(gpu, G, precision):
    """les_set_pressure_slabs(G): press_stag_array with the partitioned
    solve on the state an AB2 advance leaves (u* with its divergence), against
    the single sweep and the oracle.  FP64: 1e-12 to both.  Mixed: the two
    GPU solves differ only where the FP32 pressure spectrum rounds the
    slightly different FP64 solutions apart (1e-6), 1e-5 against the oracle
    on the same FP32-rounded inputs."""
    from new_repo_b200 import LES
    from tests.helpers import mirror, rel_err, run_params
    from tests.test_production_plans import _advance, _round_f32

    p = O.Params(nx=32, ny=32, nz=64, dt=2e-4)
    ops, st = _advance(p)
    gst = st.copy()
    if precision == "mixed":
        _round_f32(gst)
    outs = {}
    for g in (1, G):
        les = LES(run_params(p), precision=precision)
        mirror(les, gst)
        les.set_pressure_slabs(g)
        les.press_stag_array(1.5)
        outs[g] = {n: les.download(n) for n in ("p", "dpdx", "dpdy", "dpdz")}
        assert les.status() == 0
        les.close()
    ost = gst.copy()  # the oracle on the same (FP32-representable in mixed) inputs
    O.press_stag_array(ops, ost, 1.5)
    for n in ("p", "dpdx", "dpdy", "dpdz"):
        a, b, o = outs[G][n], outs[1][n], getattr(ost, n)
        if n == "p":
            a, b, o = a[:-1], b[:-1], o[:-1]
        assert rel_err(a, b) <= (1e-12 if precision == "fp64" else 1e-6), (G, precision, n, rel_err(a, b))
        assert rel_err(a, o) <= (1e-12 if precision == "fp64" else 1e-5), (G, precision, n, rel_err(a, o))


@pytest.mark.gpu
def test_step_with_pressure_slabs(gpu):
    """Ten full steps with the partitioned pressure solve (4 slabs) track the
    single-sweep run to 1e-10."""
    from new_repo_b200 import LES
    from tests.helpers import rel_err, run_params

    p = O.Params(nx=32, ny=32, nz=32)
    runs = []
    for g in (1, 4):
        les = LES(run_params(p))
        les.set_initial_conditions(*O.log_law_fields(p, seed=1))
        les.set_pressure_slabs(g)
        les.step(10)
        runs.append({n: les.download(n)[1:-1] for n in ("u", "v", "w", "p")})
        les.close()
    for n in ("u", "v", "w", "p"):
        assert rel_err(runs[1][n], runs[0][n]) <= 1e-10, n


@pytest.mark.gpu
def test_pressure_slabs_reject_bad_counts(gpu):
    from new_repo_b200 import LES, LesError
    from tests.helpers import run_params

    les = LES(run_params(O.Params(nx=16, ny=16, nz=12)))
    for bad in (0, 5, 7, 12, 65):
        with pytest.raises(LesError):
            les.set_pressure_slabs(bad)
    les.set_pressure_slabs(6)
    les.close()
