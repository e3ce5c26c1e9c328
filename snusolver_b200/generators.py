"""Seeded synthetic matrices for the benchmark configurations.

The reference ships one 20x20 fixture and runs SuiteSparse matrices that are
not available here; these generators stand in for them with the shapes,
sizes and value distributions of the five workloads:

* ``laplace2d_perturbed`` -- 2D 5-point, diagonal 4*1.01, each directed
  off-diagonal -1 + U[-0.1, 0.1] (128x128, seed 0 for the plain FP64 case).
* ``convdiff3d`` -- 3D 7-point diffusion (-1 per neighbour, 6 on the
  diagonal) plus first-order upwind convection with cell Peclet 0.5 along a
  fixed unit vector (64^3).
* ``laplace2d_lognormal`` -- SPD 2D 5-point with lognormal edge weights and
  Dirichlet boundary edges (the batched 256-grid case).
* ``stencil27_lognormal`` -- 3D 27-point with lognormal(0, 2) edge weights and
  a diagonal 1.05x the row's absolute off-diagonal sum (96^3).

Random numbers come from ``numpy.random.default_rng(seed)``; values are drawn
row-major over the CSR entries (one draw per entry, used by off-diagonals).
All matrices are CSR with int32 indices, sorted columns and no duplicates.
"""
from __future__ import annotations

import numpy as np

GENERATOR_VERSION = 1


def _grid_csr(shape, offsets):
    """Pattern of a stencil on a grid (C order, last axis fastest).

    Returns (rowptr, colidx, diag_mask, offset_id) where offset_id[k] is the
    index into ``offsets`` of entry k (-1 for the diagonal).
    """
    shape = tuple(int(s) for s in shape)
    n = int(np.prod(shape))
    coords = np.stack(np.unravel_index(np.arange(n), shape), axis=1)
    rows, cols, oid = [np.arange(n)], [np.arange(n)], [np.full(n, -1)]
    for k, off in enumerate(offsets):
        nb = coords + np.asarray(off)
        ok = np.all((nb >= 0) & (nb < np.asarray(shape)), axis=1)
        r = np.nonzero(ok)[0]
        c = np.ravel_multi_index(tuple(nb[ok].T), shape)
        rows.append(r)
        cols.append(c)
        oid.append(np.full(len(r), k))
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    oid = np.concatenate(oid)
    order = np.lexsort((cols, rows))
    rows, cols, oid = rows[order], cols[order], oid[order]
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rowptr, rows + 1, 1)
    rowptr = np.cumsum(rowptr)
    return (rowptr.astype(np.int32), cols.astype(np.int32), rows.astype(np.int64),
            oid)


def _neighbours(dim, full):
    offs = []
    if full:
        for d in np.ndindex(*([3] * dim)):
            o = tuple(int(x) - 1 for x in d)
            if any(o):
                offs.append(o)
    else:
        for a in range(dim):
            for s in (-1, 1):
                o = [0] * dim
                o[a] = s
                offs.append(tuple(o))
    return offs


def laplace2d_perturbed(nx=128, ny=128, seed=0):
    """2D 5-point Laplacian, diagonal 4*1.01, off-diagonals -1 + U[-0.1,0.1]."""
    offs = _neighbours(2, False)
    rowptr, colidx, rows, oid = _grid_csr((nx, ny), offs)
    rng = np.random.default_rng(seed)
    u = rng.uniform(-0.1, 0.1, size=len(colidx))
    vals = np.where(oid < 0, 4.0 * 1.01, -1.0 + u)
    return rowptr, colidx, vals.astype(np.float64)


CONVDIFF_DIRECTION = np.array([1.0, 2.0, 3.0]) / np.sqrt(14.0)


def convdiff3d(n=64, peclet=0.5, direction=CONVDIFF_DIRECTION):
    """3D 7-point diffusion + first-order upwind convection.

    Diffusion: -1 per neighbour, 6 on the diagonal.  Convection velocity
    b = 2*Pe*direction (cell Peclet Pe with unit spacing and diffusivity);
    for b_d > 0 the upwind neighbour is the one at -1 along axis d: it gets
    -b_d and the diagonal +b_d (mirrored for b_d < 0).  Boundary neighbours
    are dropped (Dirichlet truncation).
    """
    offs = _neighbours(3, False)
    rowptr, colidx, rows, oid = _grid_csr((n, n, n), offs)
    b = 2.0 * peclet * np.asarray(direction, dtype=np.float64)
    vals = np.full(len(colidx), -1.0)
    diag = 6.0 + np.abs(b).sum()
    vals[oid < 0] = diag
    for k, off in enumerate(offs):
        axis = int(np.nonzero(off)[0][0])
        sgn = off[axis]
        upwind = (b[axis] > 0 and sgn < 0) or (b[axis] < 0 and sgn > 0)
        if upwind:
            vals[oid == k] -= abs(b[axis])
    return rowptr, colidx, vals


def laplace2d_lognormal(nx, ny, seed, sigma=1.0):
    """SPD 2D 5-point: symmetric edge weights w~lognormal(0, sigma),
    off-diagonal -w, diagonal = sum of incident weights including virtual
    Dirichlet edges to the boundary (each also lognormal)."""
    rng = np.random.default_rng(seed)
    # horizontal edges (x, y)-(x+1, y) and vertical (x, y)-(x, y+1), plus
    # boundary edges on all four sides
    wh = rng.lognormal(0.0, sigma, size=(nx + 1, ny))
    wv = rng.lognormal(0.0, sigma, size=(nx, ny + 1))
    offs = _neighbours(2, False)  # (-1,0),(1,0),(0,-1),(0,1)
    rowptr, colidx, rows, oid = _grid_csr((nx, ny), offs)
    xs, ys = np.unravel_index(rows, (nx, ny))
    vals = np.zeros(len(colidx))
    w = [wh[xs, ys], wh[xs + 1, ys], wv[xs, ys], wv[xs, ys + 1]]
    for k in range(4):
        m = oid == k
        vals[m] = -w[k][m]
    dm = oid < 0
    xd, yd = xs[dm], ys[dm]
    vals[dm] = wh[xd, yd] + wh[xd + 1, yd] + wv[xd, yd] + wv[xd, yd + 1]
    return rowptr, colidx, vals


def laplace3d_lognormal(nx, ny, nz, seed, sigma=1.0):
    """SPD 3D 7-point: symmetric edge weights lognormal(0, sigma) (one per
    grid edge, boundary edges to the Dirichlet boundary included in the
    diagonal), off-diagonal -w, diagonal = sum of incident weights."""
    rng = np.random.default_rng(seed)
    shape = (nx, ny, nz)
    offs = _neighbours(3, False)  # (-1,0,0),(1,0,0),(0,-1,0),(0,1,0),...
    rowptr, colidx, rows, oid = _grid_csr(shape, offs)
    # weights of the edges between x and x+1 along each axis (boundary
    # edges at both ends included): shape + 1 along that axis
    w = [rng.lognormal(0.0, sigma, size=tuple(s + (a == k) for k, s in
                                             enumerate(shape)))
         for a in range(3)]
    co = np.unravel_index(rows, shape)
    vals = np.zeros(len(colidx))
    for k, off in enumerate(offs):
        a = int(np.nonzero(off)[0][0])
        m = oid == k
        idx = [c[m] for c in co]
        if off[a] > 0:
            idx[a] = idx[a] + 1
        vals[m] = -w[a][tuple(idx)]
    dm = oid < 0
    d = np.zeros(int(dm.sum()))
    idx = [c[dm] for c in co]
    for a in range(3):
        lo = list(idx)
        hi = list(idx)
        hi[a] = hi[a] + 1
        d += w[a][tuple(lo)] + w[a][tuple(hi)]
    vals[dm] = d
    return rowptr, colidx, vals


def stencil27_lognormal(n=96, seed=4, sigma=2.0):
    """3D 27-point, symmetric edge weights lognormal(0, sigma) (off-diagonal
    -w), diagonal 1.05 x the row's absolute off-diagonal sum."""
    offs = _neighbours(3, True)
    rowptr, colidx, rows, oid = _grid_csr((n, n, n), offs)
    rng = np.random.default_rng(seed)
    # one weight per undirected edge: key by (min, max)
    lo = np.minimum(rows, colidx.astype(np.int64))
    hi = np.maximum(rows, colidx.astype(np.int64))
    off = oid >= 0
    keys = lo[off] * (n ** 3) + hi[off]
    uk, inv = np.unique(keys, return_inverse=True)
    w = rng.lognormal(0.0, sigma, size=len(uk))
    vals = np.zeros(len(colidx))
    vals[off] = -w[inv]
    rowsum = np.zeros(n ** 3)
    np.add.at(rowsum, rows[off], np.abs(vals[off]))
    vals[~off] = 1.05 * rowsum[rows[~off]]
    return rowptr, colidx, vals, rng


def batch_config(name="c3_batch256", count=256, seed=3, lo=32, hi=256):
    """The batched workload: `count` independent SPD 2D 5-point matrices,
    grid sides drawn uniformly from lo..hi per axis (seed 3), edge weights
    lognormal(0, 1).  Returns a list of (rowptr, colidx, vals)."""
    if name != "c3_batch256":
        raise KeyError(name)
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, size=(count, 2))
    return [laplace2d_lognormal(int(nx), int(ny), seed=seed * 1000 + k)
            for k, (nx, ny) in enumerate(sides)]


def rhs(n, nrhs, seed, lo=-1.0, hi=1.0):
    """Column-major (n, nrhs) right-hand sides U[lo, hi]."""
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.uniform(lo, hi, size=(nrhs, n)).T)


def write_mtx(path, rowptr, colidx, vals, comment="snusolver_b200 generator"):
    """MatrixMarket coordinate real general, entries in CSR order."""
    rowptr = np.asarray(rowptr)
    n = len(rowptr) - 1
    rows = np.repeat(np.arange(n), np.diff(rowptr))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"% {comment}\n")
        f.write(f"{n} {n} {len(colidx)}\n")
        data = np.column_stack([rows + 1, np.asarray(colidx) + 1,
                                np.asarray(vals)])
        np.savetxt(f, data, fmt=["%d", "%d", "%.17g"])


def config(name):
    """(rowptr, colidx, vals, B) of a named workload."""
    if name == "c1_2d128":
        rp, ci, v = laplace2d_perturbed(128, 128, seed=0)
        return rp, ci, v, rhs(len(rp) - 1, 1, seed=1)
    if name == "c2_convdiff64":
        rp, ci, v = convdiff3d(64)
        return rp, ci, v, rhs(len(rp) - 1, 4, seed=2)
    if name == "c4_27pt96":
        rp, ci, v, rng = stencil27_lognormal(96, seed=4)
        n = len(rp) - 1
        B = np.asfortranarray(rng.uniform(-1.0, 1.0, size=(16, n)).T)
        return rp, ci, v, B
    if name.startswith("convdiff") and name[8:].isdigit():
        m = int(name[8:])
        rp, ci, v = convdiff3d(m)
        return rp, ci, v, rhs(len(rp) - 1, 4, seed=2)
    raise KeyError(name)


if __name__ == "__main__":
    # python -m snusolver_b200.generators NAME OUT.mtx [RHS.bin]
    # writes a named workload as MatrixMarket (and its right-hand sides as
    # raw column-major float64) for the driver or the reference's driver
    import sys
    if len(sys.argv) < 3:
        sys.exit("usage: python -m snusolver_b200.generators "
                 "{c1_2d128|c2_convdiff64|c4_27pt96|convdiffN} OUT.mtx [RHS.bin]")
    rp, ci, v, B = config(sys.argv[1])
    write_mtx(sys.argv[2], rp, ci, v, comment=f"snusolver_b200 {sys.argv[1]}")
    if len(sys.argv) > 3:
        np.asfortranarray(B).T.astype(np.float64).tofile(sys.argv[3])
