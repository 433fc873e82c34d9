"""Seeded synthetic SPD systems with the shapes the benchmarks and tests use.

  poisson7(L)          3-D 7-point Poisson, Dirichlet boundary (diag 6, off -1)
  stencil_grf(L, ...)  3-D 7/27-point variable-coefficient diffusion whose
                       cell log-coefficients g are a Gaussian random field;
                       the diagonal is the off-diagonal row sum plus a shift
  unstructured(L, ...) 7-point graph with a fraction of face pairs removed,
                       random weights, a random symmetric permutation and a
                       diagonal of (1 + eps) times the row sum
  random_csr(...)      irregular matrices for format-conversion tests

All generators are numpy-vectorised and deterministic for a given seed.
"""
from __future__ import annotations

import numpy as np

from . import csr_matrix


def _offsets(points: int):
    offs = []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                m = abs(dx) + abs(dy) + abs(dz)
                if points == 7 and m > 1:
                    continue
                offs.append((dz, dy, dx, m))
    return offs  # sorted by linear offset dz*L*L + dy*L + dx


def _assemble(L: int, points: int, weight_fn, diag_fn):
    """CSR of a box stencil.  weight_fn(idx_i, idx_j, m) gives the coupling
    weight (positive) of the listed neighbour pairs; the off-diagonal entry is
    its negative.  diag_fn(rowsum) gives the diagonal."""
    n = L * L * L
    idx = np.arange(n, dtype=np.int64)
    z, y, x = idx // (L * L), (idx // L) % L, idx % L
    offs = _offsets(points)
    k = len(offs)
    cols = np.empty((n, k), np.int64)
    vals = np.zeros((n, k), np.float64)
    valid = np.zeros((n, k), bool)
    rowsum = np.zeros(n)
    dpos = None
    for c, (dz, dy, dx, m) in enumerate(offs):
        if m == 0:
            dpos = c
            cols[:, c] = idx
            valid[:, c] = True
            continue
        ok = ((z + dz >= 0) & (z + dz < L) & (y + dy >= 0) & (y + dy < L) &
              (x + dx >= 0) & (x + dx < L))
        j = idx + dz * L * L + dy * L + dx
        cols[:, c] = np.where(ok, j, 0)
        w = np.zeros(n)
        w[ok] = weight_fn(idx[ok], j[ok], m)
        vals[:, c] = -w
        valid[:, c] = ok
        rowsum += w
    vals[:, dpos] = diag_fn(rowsum)
    counts = valid.sum(1)
    row_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    return csr_matrix(n, n, row_ptr.astype(np.int32), cols[valid].astype(np.int32),
                      vals[valid])


def poisson7(L: int) -> csr_matrix:
    """7-point Poisson, Dirichlet: 6 on the diagonal, -1 to each in-grid face
    neighbour (the operator of a 32^3 grid has 223,232 non-zeros)."""
    return _assemble(L, 7, lambda i, j, m: np.ones(i.shape), lambda s: np.full(s.shape, 6.0))


def gaussian_random_field(L: int, corr_len: float, sigma: float, seed: int) -> np.ndarray:
    """Periodic Gaussian random field on an L^3 grid: white noise smoothed by
    a Gaussian kernel exp(-r^2 / (2 corr_len^2)) in Fourier space, rescaled to
    zero mean and standard deviation sigma."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((L, L, L))
    k = np.fft.fftfreq(L) * 2 * np.pi
    kz, ky, kx = np.meshgrid(k, k, k[: L // 2 + 1], indexing="ij")
    filt = np.exp(-0.5 * (corr_len ** 2) * (kx ** 2 + ky ** 2 + kz ** 2))
    g = np.fft.irfftn(np.fft.rfftn(w) * filt, s=(L, L, L), axes=(0, 1, 2))
    g -= g.mean()
    s = g.std()
    return (g / (s if s > 0 else 1.0) * sigma).ravel()


def stencil_grf(L: int, points: int = 27, corr_len: float = 8.0, sigma: float = 1.5,
                seed: int = 0, shift: float = 1e-3) -> csr_matrix:
    """Variable-coefficient diffusion: the coupling of cells i and j is
    exp((g_i + g_j) / 2) / d_ij^2 (d^2 = 1 face, 2 edge, 3 corner neighbours),
    g a Gaussian random field; diagonal = row sum of couplings + shift, so the
    matrix is an SPD M-matrix."""
    g = gaussian_random_field(L, corr_len, sigma, seed)
    return _assemble(L, points, lambda i, j, m: np.exp(0.5 * (g[i] + g[j])) / m,
                     lambda s: s + shift)


def lognormal_stencil(L, points, sigma, seed, shift=1e-3, dims=None) -> csr_matrix:
    """Box stencil with independent log-normal couplings exp(N(0, sigma^2))
    per pair (symmetric), diagonal = row sum + shift."""
    if dims is not None and not (dims[0] == dims[1] == dims[2]):
        return _box_lognormal(dims, points, sigma, seed, shift)
    rng = np.random.default_rng(seed)
    n = L * L * L
    cell = rng.standard_normal(n) * sigma
    return _assemble(L, points, lambda i, j, m: np.exp(0.5 * (cell[i] + cell[j])), lambda s: s + shift)


def _box_lognormal(dims, points, sigma, seed, shift):
    nz, ny, nx = dims
    n = nz * ny * nx
    rng = np.random.default_rng(seed)
    cell = rng.standard_normal(n) * sigma
    idx = np.arange(n, dtype=np.int64)
    z, y, x = idx // (ny * nx), (idx // nx) % ny, idx % nx
    offs = _offsets(points)
    k = len(offs)
    cols = np.empty((n, k), np.int64)
    vals = np.zeros((n, k))
    valid = np.zeros((n, k), bool)
    rowsum = np.zeros(n)
    dpos = 0
    for c, (dz, dy, dx, m) in enumerate(offs):
        if m == 0:
            dpos = c
            cols[:, c] = idx
            valid[:, c] = True
            continue
        ok = ((z + dz >= 0) & (z + dz < nz) & (y + dy >= 0) & (y + dy < ny) &
              (x + dx >= 0) & (x + dx < nx))
        j = idx + dz * ny * nx + dy * nx + dx
        cols[:, c] = np.where(ok, j, 0)
        w = np.zeros(n)
        w[ok] = np.exp(0.5 * (cell[idx[ok]] + cell[j[ok]]))
        vals[:, c] = -w
        valid[:, c] = ok
        rowsum += w
    vals[:, dpos] = rowsum + shift
    counts = valid.sum(1)
    row_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    return csr_matrix(n, n, row_ptr.astype(np.int32), cols[valid].astype(np.int32), vals[valid])


def unstructured(L: int = 192, delete_frac: float = 0.05, seed: int = 1, wlo: float = 0.1,
                 whi: float = 10.0, diag_scale: float = 1.01) -> csr_matrix:
    """7-point face graph on an L^3 grid with delete_frac of the face pairs
    removed at random, remaining pair weights U(wlo, whi), a random symmetric
    permutation of the unknowns, diagonal = diag_scale * row sum."""
    rng = np.random.default_rng(seed)
    n = L ** 3
    idx = np.arange(n, dtype=np.int64)
    z, y, x = idx // (L * L), (idx // L) % L, idx % L
    pi, pj = [], []
    for (ok, step) in ((x + 1 < L, 1), (y + 1 < L, L), (z + 1 < L, L * L)):
        pi.append(idx[ok])
        pj.append(idx[ok] + step)
    pi = np.concatenate(pi)
    pj = np.concatenate(pj)
    keep = rng.random(pi.size) >= delete_frac
    pi, pj = pi[keep], pj[keep]
    w = rng.uniform(wlo, whi, pi.size)
    perm = rng.permutation(n)
    pi, pj = perm[pi], perm[pj]
    rows = np.concatenate([pi, pj])
    cols = np.concatenate([pj, pi])
    vals = -np.concatenate([w, w])
    rowsum = np.bincount(rows, weights=-vals, minlength=n)
    rows = np.concatenate([rows, np.arange(n)])
    cols = np.concatenate([cols, np.arange(n)])
    vals = np.concatenate([vals, diag_scale * rowsum + (rowsum == 0)])
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    row_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=n), out=row_ptr[1:])
    return csr_matrix(n, n, row_ptr.astype(np.int32), cols.astype(np.int32), vals)


def random_csr(n_rows: int, n_cols: int, seed: int, mean_len: float = 8.0,
               max_len: int = 64, pair_frac: float = 0.3, band: int | None = None,
               dtype=np.float64, empty_frac: float = 0.05) -> csr_matrix:
    """Irregular CSR with sorted unique columns: row lengths vary widely, some
    rows are empty, and about pair_frac of the entries come as aligned
    (even, odd) column pairs so that hblock extraction has something to find.
    band limits columns to |c - r| <= band (diagonal-friendly) when given."""
    rng = np.random.default_rng(seed)
    lens = np.minimum(rng.geometric(1.0 / max(mean_len, 1.0), n_rows), max_len)
    lens[rng.random(n_rows) < empty_frac] = 0
    rp = [0]
    cols_all, vals_all = [], []
    for r in range(n_rows):
        ln = int(lens[r])
        if band is not None:
            lo, hi = max(0, r - band), min(n_cols, r + band + 1)
        else:
            lo, hi = 0, n_cols
        span = hi - lo
        ln = min(ln, span)
        if ln == 0:
            rp.append(rp[-1])
            continue
        c = set()
        npair = int(ln * pair_frac) // 2
        for _ in range(npair):
            e = lo + 2 * int(rng.integers(0, max(1, span // 2)))
            if e + 1 < hi:
                c.add(e)
                c.add(e + 1)
        while len(c) < ln:
            c.add(int(lo + rng.integers(0, span)))
        c = np.array(sorted(c), np.int64)[: max(ln, 0)] if len(c) > ln else np.array(sorted(c))
        cols_all.append(c)
        vals_all.append(rng.standard_normal(c.size))
        rp.append(rp[-1] + c.size)
    cols = np.concatenate(cols_all) if cols_all else np.zeros(0, np.int64)
    vals = np.concatenate(vals_all) if vals_all else np.zeros(0)
    return csr_matrix(n_rows, n_cols, np.array(rp, np.int32), cols.astype(np.int32),
                      vals.astype(dtype))


def batch_systems(n_systems: int = 96, seed: int = 0, lo: int = 16, hi: int = 64,
                  frac7: float = 0.6, sigma: float = 1.0, rhs_lo: int = 1, rhs_hi: int = 4,
                  shift: float = 1e-3):
    """Uneven batch of independent SPD systems: each a 7-point (probability
    frac7) or 27-point box stencil with side lengths drawn uniformly from
    lo..hi per axis, independent log-normal couplings exp(N(0, sigma^2)),
    diagonal = row sum + shift, and rhs_lo..rhs_hi right-hand sides.
    Returns (systems, n_rhs, dims)."""
    rng = np.random.default_rng(seed)
    systems, n_rhs, dims = [], [], []
    for k in range(n_systems):
        d = tuple(int(v) for v in rng.integers(lo, hi + 1, size=3))
        points = 7 if rng.random() < frac7 else 27
        r = int(rng.integers(rhs_lo, rhs_hi + 1))
        systems.append(_box_lognormal(d, points, sigma, seed * 1000 + k, shift))
        n_rhs.append(r)
        dims.append(d + (points,))
    return systems, n_rhs, dims


def batch_rhs(systems, n_rhs, seed: int = 0):
    """x_true ~ U(-1, 1) per (system, rhs) and b = A x_true, as arrays of
    shape (n_rhs[k], n_k)."""
    rng = np.random.default_rng(seed)
    xs, bs = [], []
    for A, r in zip(systems, n_rhs):
        S = A.to_scipy()
        x = rng.uniform(-1.0, 1.0, size=(r, A.n_rows))
        xs.append(x)
        bs.append(np.ascontiguousarray((S @ x.T).T))
    return xs, bs
