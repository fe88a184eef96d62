"""z-slab decomposition over torch.distributed: the ghost-plane exchange and
the partitioned tridiagonal pressure solve, rank by rank.

A rank of G holds global levels r m + 1 .. (r+1) m of every field (m = nz/G)
as a (m + 2, ny, nx) array with one ghost level on each side, the layout of
the one-domain state.  The reference's 2DECOMP&FFT decomposition refreshes
ghosts with update_ghost / update_halo3 (decomp_2d_custom.f90:324-473,
902-1024) and transposes the pressure's spectral right-hand side from
z-slabs to columns and back around the tridiagonal solve
(compute_pressure.f90:265,290).  Here:

* halo_exchange: each rank sends its top interior level up and its bottom
  interior level down (one plane per neighbour, point to point); the end
  ranks keep their physical ghosts.
* partitioned_solve: each rank eliminates its own rows of every (kx, ky)
  column with three right-hand sides (the right-hand side and the unit
  couplings to the neighbours' boundary unknowns), the six boundary values
  per column are all-gathered, every rank solves the 2G-unknown reduced
  system (2 x 2 block Thomas) redundantly and back-substitutes its rows.
  Traffic per rank: 2 x 6 values per column instead of a full transpose.

The tensors may live on the CPU (gloo) or on a GPU (NCCL); the arithmetic is
torch's, so the same code is the host logic tested over gloo and the data
path between GPUs.  Complex tensors cross the collectives as real views.
"""
from __future__ import annotations

import torch


def slab_rows(nz: int, G: int, rank: int) -> tuple[int, int]:
    """Rows (start, end) of the pressure columns (rows 0..nz+1) held by
    `rank`: its levels, plus the bottom row on rank 0 and the top row on
    the last rank."""
    if G < 1 or nz % G:
        raise ValueError("nz must be a multiple of the number of slabs")
    m = nz // G
    s = 0 if rank == 0 else rank * m + 1
    e = (rank + 1) * m if rank < G - 1 else nz + 1
    return s, e


def halo_exchange(dist, local: torch.Tensor, group=None) -> None:
    """Refresh the ghost levels 0 and m+1 of this rank's (m+2, ny, nx) slab
    from the neighbouring ranks (in place)."""
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    m = local.shape[0] - 2
    ops = []
    if rank + 1 < world:
        ops.append(dist.P2POp(dist.isend, local[m].contiguous(), rank + 1, group))
        top = torch.empty_like(local[m + 1])
        ops.append(dist.P2POp(dist.irecv, top, rank + 1, group))
    if rank > 0:
        ops.append(dist.P2POp(dist.isend, local[1].contiguous(), rank - 1, group))
        bot = torch.empty_like(local[0])
        ops.append(dist.P2POp(dist.irecv, bot, rank - 1, group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    if rank + 1 < world:
        local[m + 1].copy_(top)
    if rank > 0:
        local[0].copy_(bot)


def _local_solves(a, b, c, r, first_coupled: bool, last_coupled: bool):
    """Thomas over this rank's rows (axis 0) with the couplings to the
    neighbours moved to the right-hand side: y (for r), u (for -a_first
    e_first), v (for -c_last e_last)."""
    m = r.shape[0]
    y = torch.empty_like(r)
    u = torch.zeros_like(a)
    v = torch.zeros_like(a)
    gam = torch.zeros_like(a)
    bet = b[0].clone()
    y[0] = r[0] / bet
    if first_coupled:
        u[0] = -a[0] / bet
    if last_coupled and m == 1:
        v[0] = -c[0] / bet
    for i in range(1, m):
        gam[i] = c[i - 1] / bet
        bet = b[i] - a[i] * gam[i]
        y[i] = (r[i] - a[i] * y[i - 1]) / bet
        u[i] = (-a[i] * u[i - 1]) / bet
        rv = -c[i] if (last_coupled and i == m - 1) else 0.0
        v[i] = (rv - a[i] * v[i - 1]) / bet
    for i in range(m - 2, -1, -1):
        y[i] = y[i] - gam[i + 1] * y[i + 1]
        u[i] = u[i] - gam[i + 1] * u[i + 1]
        v[i] = v[i] - gam[i + 1] * v[i + 1]
    return y, u, v


def _reduced(ys, ye, us, ue, vs, ve):
    """2 x 2 block Thomas over the slabs (lists over ranks) -> Xs, Xe."""
    G = len(ys)
    Bp, Yp = [], []
    for k in range(G):
        b00, b01 = torch.ones_like(us[k]), torch.zeros_like(us[k])
        b10, b11 = torch.zeros_like(us[k]), torch.ones_like(us[k])
        y0, y1 = ys[k].clone(), ye[k].clone()
        if k > 0:
            p00, p01, p10, p11 = Bp[k - 1]
            det = p00 * p11 - p01 * p10
            i10, i11 = -p10 / det, p00 / det
            w0 = i10 * (-vs[k - 1]) + i11 * (-ve[k - 1])
            z = i10 * Yp[k - 1][0] + i11 * Yp[k - 1][1]
            b00 = b00 + us[k] * w0
            b10 = b10 + ue[k] * w0
            y0 = y0 + us[k] * z
            y1 = y1 + ue[k] * z
        Bp.append((b00, b01, b10, b11))
        Yp.append((y0, y1))
    Xs, Xe = [None] * G, [None] * G
    for k in range(G - 1, -1, -1):
        r0, r1 = Yp[k]
        if k < G - 1:
            r0 = r0 + vs[k] * Xs[k + 1]
            r1 = r1 + ve[k] * Xs[k + 1]
        p00, p01, p10, p11 = Bp[k]
        det = p00 * p11 - p01 * p10
        Xs[k] = (p11 * r0 - p01 * r1) / det
        Xe[k] = (-p10 * r0 + p00 * r1) / det
    return Xs, Xe


def partitioned_solve(dist, a, b, c, r, group=None) -> torch.Tensor:
    """This rank's rows x of the tridiagonal systems a x_{i-1} + b x_i +
    c x_{i+1} = r whose rows are spread over the ranks in order (axis 0 =
    this rank's rows, the other axes the columns; a, b, c real, r complex).
    Every rank takes part in the one all-gather."""
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    y, u, v = _local_solves(a, b, c, r, rank > 0, rank < world - 1)
    # the six boundary values of every column, as one real tensor
    mine = torch.stack([torch.view_as_real(y[0]).select(-1, 0), torch.view_as_real(y[0]).select(-1, 1),
                        torch.view_as_real(y[-1]).select(-1, 0), torch.view_as_real(y[-1]).select(-1, 1),
                        u[0], u[-1], v[0], v[-1]])
    got = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(got, mine.contiguous(), group=group)
    ys = [torch.complex(g[0], g[1]) for g in got]
    ye = [torch.complex(g[2], g[3]) for g in got]
    us = [g[4] for g in got]
    ue = [g[5] for g in got]
    vs = [g[6] for g in got]
    ve = [g[7] for g in got]
    Xs, Xe = _reduced(ys, ye, us, ue, vs, ve)
    xl = Xe[rank - 1] if rank > 0 else torch.zeros_like(y[0])
    xr = Xs[rank + 1] if rank < world - 1 else torch.zeros_like(y[0])
    return y + u * xl + v * xr
