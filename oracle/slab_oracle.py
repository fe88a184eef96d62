"""FP64 CPU restatement of the z-slab decomposition's two data-path pieces --
test infrastructure only (imported by tests/, never by the product path).

The reference decomposes its domain with 2DECOMP&FFT pencils: ghost planes
are exchanged by update_ghost / update_halo3 (decomp_2d_custom.f90:324-473,
902-1024) and the pressure's spectral right-hand side is transposed from
z-slabs to columns and back around the tridiagonal solve
(compute_pressure.f90:265,290).  The z-slab design solves the columns where
they lie instead, with the partition method: block b of the rows (one slab)
eliminates its own rows with three right-hand sides -- the right-hand side r
and the unit couplings to the two neighbouring slabs' boundary unknowns --
the 2 G boundary unknowns of every column solve a block-tridiagonal system of
2 x 2 blocks, and each slab back-substitutes.  In exact arithmetic the
solution is the single-sweep Thomas solution.

Rows of a column are 0..n-1 (the reference's rows 1..nz+2: bottom Neumann
row, nz interior rows, top row); slab b of G owns rows [starts[b], ends[b]]
with the boundary rows on the first and last slab, as a z-slab rank that
holds levels b nz/G + 1 .. (b+1) nz/G would.
"""
from __future__ import annotations

import numpy as np


def slab_rows(nz: int, G: int):
    """(start, end) row ranges of the G slabs of a column of nz + 2 rows."""
    if G < 1 or nz % G:
        raise ValueError("nz must be a multiple of the slab count")
    m = nz // G
    out = []
    for b in range(G):
        s = 0 if b == 0 else b * m + 1
        e = (b + 1) * m if b < G - 1 else nz + 1
        out.append((s, e))
    return out


def local_solves(a, b, c, r, s, e):
    """Thomas on rows s..e with the couplings a_s x_{s-1} and c_e x_{e+1}
    moved to the right: y (for r), u (for -a_s e_first), v (for -c_e e_last).
    a, b, c: (n, ...) real; r: (n, ...) complex; returns y, u, v over the rows."""
    m = e - s + 1
    shp = r.shape[1:]
    y = np.zeros((m,) + shp, dtype=r.dtype)
    u = np.zeros((m,) + shp)
    v = np.zeros((m,) + shp)
    gam = np.zeros((m,) + shp)
    bet = b[s].copy()
    y[0] = r[s] / bet
    u[0] = (-a[s] if s > 0 else 0.0 * a[s]) / bet
    v[0] = (-c[e] if (m == 1 and e < len(a) - 1) else 0.0 * a[s]) / bet
    for i in range(1, m):
        k = s + i
        gam[i] = c[k - 1] / bet
        bet = b[k] - a[k] * gam[i]
        y[i] = (r[k] - a[k] * y[i - 1]) / bet
        u[i] = (0.0 - a[k] * u[i - 1]) / bet
        rv = -c[e] if (i == m - 1 and e < len(a) - 1) else 0.0
        v[i] = (rv - a[k] * v[i - 1]) / bet
    for i in range(m - 2, -1, -1):
        y[i] = y[i] - gam[i + 1] * y[i + 1]
        u[i] = u[i] - gam[i + 1] * u[i + 1]
        v[i] = v[i] - gam[i + 1] * v[i + 1]
    return y, u, v


def reduced_solve(ys, ye, us, ue, vs, ve):
    """The boundary unknowns (X_s, X_e) of every slab: for slab b,
    X_s^b - us^b X_e^{b-1} - vs^b X_s^{b+1} = ys^b and likewise for X_e^b,
    as block-Thomas elimination over 2 x 2 blocks.  Inputs are lists over the
    slabs of arrays over the columns; returns lists Xs, Xe."""
    G = len(ys)
    # Z_b = (X_s^b, X_e^b); A_b Z_{b-1} + Z_b + C_b Z_{b+1} = Y_b with
    # A_b = [[0, -us], [0, -ue]], C_b = [[-vs, 0], [-ve, 0]]
    Bp, Yp = [], []
    for b in range(G):
        B = [[np.ones_like(us[b]), np.zeros_like(us[b])], [np.zeros_like(us[b]), np.ones_like(us[b])]]
        Y = [ys[b].copy(), ye[b].copy()]
        if b > 0:
            # B_b -= A_b Bp_{b-1}^-1 C_{b-1};  Y_b -= A_b Bp_{b-1}^-1 Yp_{b-1}
            P = Bp[b - 1]
            det = P[0][0] * P[1][1] - P[0][1] * P[1][0]
            inv = [[P[1][1] / det, -P[0][1] / det], [-P[1][0] / det, P[0][0] / det]]
            # only the second component of Z_{b-1} couples: row 1 of inv
            C = [[-vs[b - 1], 0.0 * us[b]], [-ve[b - 1], 0.0 * us[b]]]
            w0 = inv[1][0] * C[0][0] + inv[1][1] * C[1][0]  # (inv C)[1][0]
            z = inv[1][0] * Yp[b - 1][0] + inv[1][1] * Yp[b - 1][1]  # (inv Y)[1]
            A = [-us[b], -ue[b]]
            B[0][0] = B[0][0] - A[0] * w0
            B[1][0] = B[1][0] - A[1] * w0
            Y[0] = Y[0] - A[0] * z
            Y[1] = Y[1] - A[1] * z
        Bp.append(B)
        Yp.append(Y)
    Xs = [None] * G
    Xe = [None] * G
    for b in range(G - 1, -1, -1):
        R = [Yp[b][0].copy(), Yp[b][1].copy()]
        if b < G - 1:
            # - C_b Z_{b+1}: only the first component of Z_{b+1}
            R[0] = R[0] + vs[b] * Xs[b + 1]
            R[1] = R[1] + ve[b] * Xs[b + 1]
        P = Bp[b]
        det = P[0][0] * P[1][1] - P[0][1] * P[1][0]
        Xs[b] = (P[1][1] * R[0] - P[0][1] * R[1]) / det
        Xe[b] = (-P[1][0] * R[0] + P[0][0] * R[1]) / det
    return Xs, Xe


def partitioned_solve(a, b, c, r, G: int):
    """x of the tridiagonal systems (rows 0..n-1 along axis 0) by the
    partition method over G slabs."""
    n = a.shape[0]
    rows = slab_rows(n - 2, G)
    with np.errstate(divide="ignore", invalid="ignore"):  # the singular Nyquist columns (skipped by callers)
        return _partitioned(a, b, c, r, G, rows)


def _partitioned(a, b, c, r, G, rows):
    parts = [local_solves(a, b, c, r, s, e) for s, e in rows]
    ys = [p[0][0] for p in parts]
    ye = [p[0][-1] for p in parts]
    us = [p[1][0] for p in parts]
    ue = [p[1][-1] for p in parts]
    vs = [p[2][0] for p in parts]
    ve = [p[2][-1] for p in parts]
    Xs, Xe = reduced_solve(ys, ye, us, ue, vs, ve)
    x = np.zeros_like(r)
    for bi, ((s, e), (y, u, v)) in enumerate(zip(rows, parts)):
        xl = Xe[bi - 1] if bi > 0 else 0.0
        xr = Xs[bi + 1] if bi < G - 1 else 0.0
        x[s:e + 1] = y + u * xl + v * xr
    return x


def halo_planes(field, G: int):
    """The ghost planes each slab of a (nz+2, ny, nx) field receives from its
    neighbours: slab b (levels b m + 1 .. (b+1) m) gets level b m below and
    level (b+1) m + 1 above, the one-domain field's neighbours (the
    physical ghost levels 0 and nz+1 on the end slabs)."""
    nz = field.shape[0] - 2
    m = nz // G
    return [(field[b * m].copy(), field[(b + 1) * m + 1].copy()) for b in range(G)]
