"""Seeded synthetic matrices of the shapes the PSBLAS drivers and the
benchmark configurations use.  Host-side (numpy), vectorised; every
generator returns a CSR triple (irp, ja, val) with 1-based int32 indices,
rows sorted by column (the order psb_spasb leaves after fix_coo), FP64
values.

* pde3d          -- the convection-diffusion operator of
                    test/pargen/psb_d_pde3d.F90:104-164,478-571 and
                    test/cudakern/dpdegenmv.F90:88-130 (7 entries per interior
                    row, Dirichlet boundary moved to the right-hand side, grid
                    step h = 1/(idim+1), index = ix + (iy-1)*n + (iz-1)*n^2 as
                    util/psb_partidx_mod.F90 ijk2idx with column-major order).
* stencil27      -- 27-point Poisson stencil (26 neighbours at -1, diagonal 26).
* poisson7       -- SPD 7-point Poisson (diagonal 6, neighbours -1).
* aniso2d        -- 2-D 5-point -eps*u_xx - u_yy (diagonal 2*eps+2).
* powerlaw       -- unstructured: per row k ~ P(k) ~ k^-alpha on [kmin,kmax]
                    off-diagonal columns uniform without repeats, values
                    N(0,1), diagonal = row abs sum + 1.
"""
from __future__ import annotations

import numpy as np


def _csr_from_offsets(n_rows, cols_list, vals_list):
    """cols_list/vals_list: per-stencil-point arrays of shape (n_rows,) with
    column -1 marking a missing neighbour; stencil points are given in
    ascending column order, so the result is column-sorted per row."""
    cols = np.stack(cols_list, axis=1)
    vals = np.stack(vals_list, axis=1)
    mask = cols >= 0
    counts = mask.sum(axis=1)
    irp = np.zeros(n_rows + 1, np.int64)
    np.cumsum(counts, out=irp[1:])
    ja = (cols[mask] + 1).astype(np.int32)
    va = vals[mask].astype(np.float64)
    return (irp + 1).astype(np.int32), ja, va


def _grid_rows(n, dims):
    idx = np.arange(n ** dims, dtype=np.int64)
    coords = []
    for _ in range(dims):
        coords.append(idx % n)
        idx = idx // n
    return coords  # x fastest


def pde3d(idim, a=(1.0, 1.0, 1.0), b=(0.0, 0.0, 0.0), c=0.0):
    """-div(a grad u) + b.grad u + c u on the unit cube, 7-point central
    differences; returns (irp, ja, val).  Coefficients are constants (the
    reference's a1..a3, b1..b3, c functions are constants in both drivers).
    Entry values are formed with the reference's expressions:
      (x-1): -a1/h^2 - b1/(2h)   (x+1): -a1/h^2 + b1/(2h)
      diag : 2*(a1+a2+a3)/h^2 + c."""
    n = int(idim)
    N = n ** 3
    h = 1.0 / (n + 1)
    sq = h * h
    h2 = 2.0 * h
    a1, a2, a3 = (float(v) for v in a)
    b1, b2, b3 = (float(v) for v in b)
    ix, iy, iz = _grid_rows(n, 3)
    row = np.arange(N, dtype=np.int64)
    full = lambda v: np.full(N, v, np.float64)
    pts = [  # ascending column order
        (iz > 0, row - n * n, -a3 / sq - b3 / h2),
        (iy > 0, row - n, -a2 / sq - b2 / h2),
        (ix > 0, row - 1, -a1 / sq - b1 / h2),
        (np.ones(N, bool), row, (2.0 * (a1 + a2 + a3)) / sq + c),
        (ix < n - 1, row + 1, -a1 / sq + b1 / h2),
        (iy < n - 1, row + n, -a2 / sq + b2 / h2),
        (iz < n - 1, row + n * n, -a3 / sq + b3 / h2),
    ]
    cols = [np.where(m, cc, -1) for m, cc, _ in pts]
    vals = [full(v) for _, _, v in pts]
    return _csr_from_offsets(N, cols, vals)


def stencil27(n):
    n = int(n)
    N = n ** 3
    ix, iy, iz = _grid_rows(n, 3)
    row = np.arange(N, dtype=np.int64)
    cols, vals = [], []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ok = ((ix + dx >= 0) & (ix + dx < n) & (iy + dy >= 0) & (iy + dy < n)
                      & (iz + dz >= 0) & (iz + dz < n))
                cols.append(np.where(ok, row + dx + dy * n + dz * n * n, -1))
                vals.append(np.full(N, 26.0 if (dx, dy, dz) == (0, 0, 0) else -1.0))
    return _csr_from_offsets(N, cols, vals)


def poisson7(n):
    n = int(n)
    N = n ** 3
    ix, iy, iz = _grid_rows(n, 3)
    row = np.arange(N, dtype=np.int64)
    pts = [(iz > 0, row - n * n, -1.0), (iy > 0, row - n, -1.0), (ix > 0, row - 1, -1.0),
           (np.ones(N, bool), row, 6.0),
           (ix < n - 1, row + 1, -1.0), (iy < n - 1, row + n, -1.0), (iz < n - 1, row + n * n, -1.0)]
    return _csr_from_offsets(N, [np.where(m, c, -1) for m, c, _ in pts], [np.full(N, v) for _, _, v in pts])


def aniso2d(n, eps):
    n = int(n)
    N = n * n
    ix, iy = _grid_rows(n, 2)
    row = np.arange(N, dtype=np.int64)
    pts = [(iy > 0, row - n, -1.0), (ix > 0, row - 1, -eps), (np.ones(N, bool), row, 2.0 * eps + 2.0),
           (ix < n - 1, row + 1, -eps), (iy < n - 1, row + n, -1.0)]
    return _csr_from_offsets(N, [np.where(m, c, -1) for m, c, _ in pts], [np.full(N, float(v)) for _, _, v in pts])


def powerlaw_lengths(nrows, alpha=2.1, kmin=1, kmax=4096, rng=None):
    rng = np.random.default_rng(0) if rng is None else rng
    k = np.arange(kmin, kmax + 1, dtype=np.float64)
    p = k ** (-alpha)
    cdf = np.cumsum(p / p.sum())
    u = rng.random(nrows)
    return (np.searchsorted(cdf, u, side="right") + kmin).clip(kmin, kmax).astype(np.int64)


def powerlaw(nrows, alpha=2.1, kmin=1, kmax=4096, seed=0):
    """Unstructured SPD-by-dominance matrix: k_i off-diagonal entries per row
    (k_i ~ power law), columns uniform without repeats and != i, values
    N(0,1); the diagonal is (row abs sum + 1)."""
    rng = np.random.default_rng(seed)
    n = int(nrows)
    k = np.minimum(powerlaw_lengths(n, alpha, kmin, kmax, rng), n - 1)
    rows = np.repeat(np.arange(n, dtype=np.int64), k)
    cols = rng.integers(0, n - 1, size=rows.size, dtype=np.int64)
    cols = cols + (cols >= rows)  # skip the diagonal
    # remove repeats within a row, redraw until every row has k distinct columns
    for _ in range(64):
        key = rows * n + cols
        order = np.argsort(key, kind="stable")
        key_s = key[order]
        dup = np.zeros(key_s.size, bool)
        dup[1:] = key_s[1:] == key_s[:-1]
        if not dup.any():
            break
        bad = order[dup]
        newc = rng.integers(0, n - 1, size=bad.size, dtype=np.int64)
        cols[bad] = newc + (newc >= rows[bad])
    vals = rng.standard_normal(rows.size)
    # add the diagonal
    absum = np.bincount(rows, weights=np.abs(vals), minlength=n)
    rows = np.concatenate([rows, np.arange(n, dtype=np.int64)])
    cols = np.concatenate([cols, np.arange(n, dtype=np.int64)])
    vals = np.concatenate([vals, absum + 1.0])
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    counts = np.bincount(rows, minlength=n)
    irp = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=irp[1:])
    return (irp + 1).astype(np.int32), (cols + 1).astype(np.int32), vals.astype(np.float64)


def powerlaw_spd(nrows, alpha=2.1, kmin=1, kmax=4096, seed=0):
    """Symmetric positive definite unstructured matrix with power-law row
    lengths: the off-diagonal pattern of `powerlaw` (k_i uniform columns per
    row, values N(0,1)) is symmetrised, B + B^T, and the diagonal is set to
    (row abs sum + 1), which makes it SPD by diagonal dominance."""
    irp, ja, va = powerlaw(nrows, alpha, kmin, kmax, seed)
    n = len(irp) - 1
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(irp.astype(np.int64)))
    cols = ja.astype(np.int64) - 1
    off = rows != cols
    r, c, v = rows[off], cols[off], va[off]
    rr = np.concatenate([r, c])
    cc = np.concatenate([c, r])
    vv = np.concatenate([v, v])
    key = rr * n + cc
    order = np.argsort(key, kind="stable")
    key, vv = key[order], vv[order]
    uniq, start = np.unique(key, return_index=True)
    vals = np.add.reduceat(vv, start)
    rr, cc = uniq // n, uniq % n
    absum = np.bincount(rr, weights=np.abs(vals), minlength=n)
    rr = np.concatenate([rr, np.arange(n, dtype=np.int64)])
    cc = np.concatenate([cc, np.arange(n, dtype=np.int64)])
    vals = np.concatenate([vals, absum + 1.0])
    o = np.lexsort((cc, rr))
    rr, cc, vals = rr[o], cc[o], vals[o]
    irp2 = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(rr, minlength=n), out=irp2[1:])
    return (irp2 + 1).astype(np.int32), (cc + 1).astype(np.int32), vals


def sort_rows_by_length(irp, ja, val):
    """Symmetric permutation P A P^T with rows (and columns) ordered by
    decreasing row length (stable).  Keeps an SPD matrix SPD; solves of the
    permuted system give the permuted solution.  Returns (irp, ja, val,
    order) with new row i = old row order[i]."""
    n = len(irp) - 1
    lens = np.diff(irp.astype(np.int64))
    order = np.argsort(-lens, kind="stable")
    inv = np.empty(n, np.int64)
    inv[order] = np.arange(n)
    rows_old = np.repeat(np.arange(n), lens)
    new_rows = inv[rows_old]
    new_cols = inv[ja.astype(np.int64) - 1]
    o = np.lexsort((new_cols, new_rows))
    counts = np.bincount(new_rows, minlength=n)
    nirp = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=nirp[1:])
    return ((nirp + 1).astype(np.int32), (new_cols[o] + 1).astype(np.int32),
            np.asarray(val, np.float64)[o], order)


def csr_to_coo(irp, ja, val):
    n = len(irp) - 1
    counts = np.diff(irp.astype(np.int64))
    ia = np.repeat(np.arange(1, n + 1, dtype=np.int32), counts)
    return ia, np.asarray(ja, np.int32), np.asarray(val, np.float64)


def csr_matvec(irp, ja, val, x):
    """y = A x in float64 with numpy (pairwise order); a quick host check,
    not the parity oracle."""
    n = len(irp) - 1
    ia, _, _ = csr_to_coo(irp, ja, val)
    return np.bincount(ia - 1, weights=val * x[ja - 1], minlength=n)
