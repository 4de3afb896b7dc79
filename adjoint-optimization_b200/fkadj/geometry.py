"""Grid geometry and objective generators (host side, O(n) once per problem).

The reference ships its generated grid and objective files
(src/cuda/data/lap_Cfile_2nd_order_grad_dx_0p035_N_256_hole_dens_16.mat,
src/cuda/data/S_1o4_N_256_hole_dens_16.mat) but not the code that made them.
The rules restated here reproduce those files exactly:

* ``active_index``: dense int32 grid, 1-based compact index of each active
  cell in increasing linear-index order (k = i*ncols + j), 0 at holes
  (consumed by num2nan, src/cuda/fk_grad_Et_mono_PARAMETERS.cu:1533-1541);
* ``ghost_lr``: per active cell, -1 when the cell above (i-1) is a hole or
  off-grid, +1 when the cell below (i+1) is, else 0 -- the direction of the
  uniform field's virtual-electrode source (gh = 2*Du/h * ghost_lr,
  src/cuda/fk_grad_Et_mono_PARAMETERS.cu:1588-1595);
* ``lap``: the no-flux 5-point Laplacian with the reference kernel's mirror
  rule (src/cuda/fk_forward_Et_mono_PARAMETERS.cu:319-424), unscaled;
* ``S = Gx^T Gx + Gy^T Gy``: G is a second-order finite-difference gradient,
  not divided by h: central (+-1/2) where both neighbours are active,
  one-sided (-3/2, 2, -1/2) where only one side has two active cells, first
  order where only one neighbour exists.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def _pad(mask: np.ndarray) -> np.ndarray:
    return np.pad(mask, 2, constant_values=False)


def clean_mask(mask: np.ndarray) -> np.ndarray:
    """Deactivates active cells whose two opposite neighbours (in either
    direction) are both missing; the reference stencil turns such a cell into
    NaN.  Repeats until none is left."""
    m = mask.astype(bool).copy()
    while True:
        P = np.pad(m, 1, constant_values=False)
        up, dn = ~P[:-2, 1:-1], ~P[2:, 1:-1]
        lf, rt = ~P[1:-1, :-2], ~P[1:-1, 2:]
        bad = m & ((up & dn) | (lf & rt))
        if not bad.any():
            return m
        m &= ~bad


def active_index(mask: np.ndarray) -> np.ndarray:
    m = mask.astype(bool).ravel()
    ai = np.zeros(m.size, dtype=np.int32)
    ai[m] = np.arange(1, int(m.sum()) + 1, dtype=np.int32)
    return ai


def ghost_lr(mask: np.ndarray) -> np.ndarray:
    m = mask.astype(bool)
    P = np.pad(m, 1, constant_values=False)
    up, dn = ~P[:-2, 1:-1], ~P[2:, 1:-1]
    g = np.zeros(m.shape)
    g[up] -= 1.0
    g[dn] += 1.0
    return g[m]


def _compact_index(m):
    idx = -np.ones(m.shape, dtype=np.int64)
    idx[m] = np.arange(int(m.sum()))
    return idx


def laplacian(mask: np.ndarray) -> sp.csc_matrix:
    """Unscaled 5-point Laplacian on the active cells (n_num x n_num)."""
    m = mask.astype(bool)
    nr, nc = m.shape
    idx = _compact_index(m)
    ii, jj = np.nonzero(m)
    rows = [idx[ii, jj]]
    cols = [idx[ii, jj]]
    vals = [np.full(ii.size, -4.0)]
    P = np.pad(m, 1, constant_values=False)
    for di, dj in ((1, 0), (0, 1)):
        has_p = P[ii + 1 + di, jj + 1 + dj]
        has_m = P[ii + 1 - di, jj + 1 - dj]
        for sel, oi, oj, w in ((has_p & has_m, di, dj, 1.0), (has_p & has_m, -di, -dj, 1.0),
                               (has_p & ~has_m, di, dj, 2.0), (~has_p & has_m, -di, -dj, 2.0)):
            rows.append(idx[ii[sel], jj[sel]])
            cols.append(idx[ii[sel] + oi, jj[sel] + oj])
            vals.append(np.full(int(sel.sum()), w))
    n = int(m.sum())
    return sp.csc_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(n, n))


def _gradient(m: np.ndarray, di: int, dj: int) -> sp.csr_matrix:
    idx = _compact_index(m)
    ii, jj = np.nonzero(m)
    P = _pad(m)

    def act(o):
        return P[ii + 2 + o * di, jj + 2 + o * dj]

    p1, m1, p2, m2 = act(1), act(-1), act(2), act(-2)
    r = idx[ii, jj]
    rows, cols, vals = [], [], []

    def add(sel, offs, ws):
        for o, w in zip(offs, ws):
            rows.append(r[sel])
            cols.append(idx[ii[sel] + o * di, jj[sel] + o * dj])
            vals.append(np.full(int(sel.sum()), w))

    central = p1 & m1
    add(central, (1, -1), (0.5, -0.5))
    fwd2 = p1 & ~m1 & p2
    add(fwd2, (0, 1, 2), (-1.5, 2.0, -0.5))
    fwd1 = p1 & ~m1 & ~p2
    add(fwd1, (0, 1), (-1.0, 1.0))
    bwd2 = ~p1 & m1 & m2
    add(bwd2, (0, -1, -2), (1.5, -2.0, 0.5))
    bwd1 = ~p1 & m1 & ~m2
    add(bwd1, (0, -1), (1.0, -1.0))
    n = int(m.sum())
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(n, n))


def objective_matrix(mask: np.ndarray) -> sp.csc_matrix:
    """S = Gx^T Gx + Gy^T Gy (spatial-variation objective, symmetric)."""
    m = mask.astype(bool)
    Gx = _gradient(m, 1, 0)
    Gy = _gradient(m, 0, 1)
    S = (Gx.T @ Gx + Gy.T @ Gy).tocsc()
    S.sum_duplicates()
    S.eliminate_zeros()
    S.sort_indices()
    return S


def mean_square_matrix(n_num: int) -> sp.csc_matrix:
    """S = (2/n_num) I: with gamma = (1,0,0) and alpha = 0 the reference's
    Lcost = L0/2 becomes J = mean over active cells of u(T)^2."""
    return sp.identity(n_num, format="csc") * (2.0 / n_num)


def circles_mask(nrows: int, ncols: int, dx: float, centres, radii) -> np.ndarray:
    """Active-cell mask with circular non-conducting obstacles: a cell whose
    centre lies inside any circle is a hole."""
    yc = (np.arange(nrows) + 0.5) * dx
    xc = (np.arange(ncols) + 0.5) * dx
    Y, X = np.meshgrid(yc, xc, indexing="ij")
    hole = np.zeros((nrows, ncols), dtype=bool)
    for (cy, cx), r in zip(centres, radii):
        i0 = max(int((cy - r) / dx) - 1, 0)
        i1 = min(int((cy + r) / dx) + 2, nrows)
        j0 = max(int((cx - r) / dx) - 1, 0)
        j1 = min(int((cx + r) / dx) + 2, ncols)
        sub = (Y[i0:i1, j0:j1] - cy) ** 2 + (X[i0:i1, j0:j1] - cx) ** 2 <= r * r
        hole[i0:i1, j0:j1] |= sub
    return clean_mask(~hole)


def nan_grid(y_compact: np.ndarray, ai: np.ndarray, nvar: int = 3) -> np.ndarray:
    """Compact [u;v;w] -> dense NaN grid (num2nan, cu-G:1533-1541)."""
    n = ai.size
    n_num = int((ai > 0).sum())
    out = np.full(nvar * n, np.nan)
    act = ai > 0
    for c in range(nvar):
        out[c * n:(c + 1) * n][act] = y_compact[c * n_num:(c + 1) * n_num][ai[act] - 1]
    return out


def compact(y_grid: np.ndarray, ai: np.ndarray, nvar: int = 3) -> np.ndarray:
    """Dense NaN grid -> compact [u;v;w] (nan2num, cu-G:1543-1551)."""
    n = ai.size
    n_num = int((ai > 0).sum())
    out = np.empty(nvar * n_num)
    act = ai > 0
    for c in range(nvar):
        out[c * n_num:(c + 1) * n_num][ai[act] - 1] = y_grid[c * n:(c + 1) * n][act]
    return out


def gh_grid(ghost: np.ndarray, ai: np.ndarray, Du: float, h: float) -> np.ndarray:
    """Dense virtual-electrode vector gh = (Du*2/h)*ghost_lr, NaN at holes."""
    out = np.full(ai.size, np.nan)
    act = ai > 0
    out[act] = Du * 2 / h * np.asarray(ghost, dtype=np.float64)[ai[act] - 1]
    return out
