"""Seeded synthetic systems for the solver workloads, as 0-based CSR (int32
row pointers and columns, float64 values, columns ascending within a row).

The reference measures on SuiteSparse matrices that are not available here;
these generated systems stand in for them with the shapes, sizes and value
distributions of the five workloads:

  laplace2d(256)          2D 5-point Dirichlet Laplacian (diag 4, off -1)
  poisson3d_varcoef(128)  3D 7-point variable-coefficient Poisson, k = exp(N(0,1))
                          per face including the Dirichlet boundary faces
  convdiff3d(96)          3D cell-centred convection-diffusion, first-order upwind,
                          v = 10 (sin y, sin z, sin x) on [0, 2 pi)^3
  aniso2d_grf(512)        2D anisotropic diffusion, kappa = exp(GRF), ratio 10
  batch_systems(...)      many independent 2D 5-point / 3D 27-point SPD systems

Orderings are natural lexicographic with x fastest.  Random draws use
numpy.random.default_rng with the seeds and draw orders written below.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class CSR:
    n: int
    rowptr: np.ndarray
    colidx: np.ndarray
    val: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """FP64 y = A x (row by row, ascending column order)."""
        prod = self.val * x[self.colidx]
        return np.add.reduceat(prod, self.rowptr[:-1]) * (np.diff(self.rowptr) > 0)

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.val, self.colidx, self.rowptr), shape=(self.n, self.n))


def _from_slots(n, cols, vals, mask) -> CSR:
    """Compress (n, k) slot arrays (already in ascending column order) to CSR."""
    counts = mask.sum(axis=1)
    rowptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=rowptr[1:])
    if rowptr[-1] >= 2**31:
        raise ValueError("nnz exceeds int32")
    return CSR(n, rowptr.astype(np.int32), cols[mask].astype(np.int32), vals[mask].astype(np.float64))


def laplace2d(N: int = 256) -> CSR:
    """5-point Laplacian on an N x N grid, Dirichlet boundary: diag 4, off -1."""
    n = N * N
    idx = np.arange(n, dtype=np.int64)
    x, y = idx % N, idx // N
    cols = np.stack([idx - N, idx - 1, idx, idx + 1, idx + N], axis=1)
    mask = np.stack([y > 0, x > 0, np.ones(n, bool), x < N - 1, y < N - 1], axis=1)
    vals = np.stack([np.full(n, -1.0), np.full(n, -1.0), np.full(n, 4.0),
                     np.full(n, -1.0), np.full(n, -1.0)], axis=1)
    return _from_slots(n, cols, vals, mask)


def _streams(seed: int, k: int):
    return [np.random.default_rng(s) for s in np.random.SeedSequence(seed).spawn(k)]


def poisson3d_varcoef(N: int = 128, seed: int = 1):
    """3D 7-point variable-coefficient Poisson on N^3 cells.

    One g ~ N(0,1) per face, k_f = exp(g).  Draw order from the coefficient
    stream (SeedSequence(seed).spawn(2)[0]): interior x-faces (z, y, x-face)
    C-order, interior y-faces, interior z-faces, then the boundary faces
    x-low, x-high, y-low, y-high, z-low, z-high (N*N each, C-order).
    A = sum_f k_f (e_i - e_j)(e_i - e_j)^T + sum_boundary k_f e_i e_i^T (SPD).
    x_true ~ U(-1, 1) from the second stream; returns (A, b = A x_true, x_true).
    """
    rc, rx = _streams(seed, 2)
    kx = np.empty((N, N, N + 1))
    ky = np.empty((N, N + 1, N))
    kz = np.empty((N + 1, N, N))
    kx[:, :, 1:N] = np.exp(rc.standard_normal((N, N, N - 1)))
    ky[:, 1:N, :] = np.exp(rc.standard_normal((N, N - 1, N)))
    kz[1:N, :, :] = np.exp(rc.standard_normal((N - 1, N, N)))
    kx[:, :, 0] = np.exp(rc.standard_normal((N, N)))
    kx[:, :, N] = np.exp(rc.standard_normal((N, N)))
    ky[:, 0, :] = np.exp(rc.standard_normal((N, N)))
    ky[:, N, :] = np.exp(rc.standard_normal((N, N)))
    kz[0, :, :] = np.exp(rc.standard_normal((N, N)))
    kz[N, :, :] = np.exp(rc.standard_normal((N, N)))
    n = N ** 3
    diag = (kx[:, :, :N] + kx[:, :, 1:] + ky[:, :N, :] + ky[:, 1:, :] + kz[:N] + kz[1:]).reshape(n)
    idx = np.arange(n, dtype=np.int64)
    x = idx % N
    y = (idx // N) % N
    z = idx // (N * N)
    cols = np.stack([idx - N * N, idx - N, idx - 1, idx, idx + 1, idx + N, idx + N * N], axis=1)
    mask = np.stack([z > 0, y > 0, x > 0, np.ones(n, bool), x < N - 1, y < N - 1, z < N - 1], axis=1)
    vals = np.stack([-kz[:N].reshape(n), -ky[:, :N, :].reshape(n), -kx[:, :, :N].reshape(n), diag,
                     -kx[:, :, 1:].reshape(n), -ky[:, 1:, :].reshape(n), -kz[1:].reshape(n)], axis=1)
    A = _from_slots(n, cols, vals, mask)
    x_true = rx.uniform(-1.0, 1.0, n)
    return A, A.matvec(x_true), x_true


def laplace2d_system(N: int = 256, seed: int = 0):
    """The 2D Laplacian with b = A x_true, x_true ~ U(-1,1) from default_rng(seed)."""
    A = laplace2d(N)
    x_true = np.random.default_rng(seed).uniform(-1.0, 1.0, A.n)
    return A, A.matvec(x_true), x_true


def convdiff3d(N: int = 96, seed: int = 2, vscale: float = 10.0):
    """Nonsymmetric 3D convection-diffusion, cell-centred on [0, 2 pi)^3, h = 2 pi / N.

    -Laplace(u) (unit diffusion, 7-point) + v . grad(u) with first-order upwind
    differences, v = vscale (sin y, sin z, sin x) at cell centres.  Homogeneous
    Dirichlet at the domain faces through ghost cells u_ghost = -u (a missing
    neighbour adds its coupling with the opposite sign to the diagonal).
    b = A 1 + 0.01 N(0,1) from default_rng(seed).  Returns (A, b, peclet_max).
    """
    h = 2.0 * np.pi / N
    n = N ** 3
    idx = np.arange(n, dtype=np.int64)
    x = idx % N
    y = (idx // N) % N
    z = idx // (N * N)
    xc, yc, zc = (x + 0.5) * h, (y + 0.5) * h, (z + 0.5) * h
    vx, vy, vz = vscale * np.sin(yc), vscale * np.sin(zc), vscale * np.sin(xc)
    inv_h2, inv_h = 1.0 / (h * h), 1.0 / h
    # coupling to the minus / plus neighbour along each axis (diffusion + upwind)
    def axis(v):
        cm = -inv_h2 - np.maximum(v, 0.0) * inv_h     # coefficient of u_{i-1}
        cp = -inv_h2 + np.minimum(v, 0.0) * inv_h     # coefficient of u_{i+1}
        cd = 2.0 * inv_h2 + np.abs(v) * inv_h         # diagonal part
        return cm, cp, cd
    cmx, cpx, cdx = axis(vx)
    cmy, cpy, cdy = axis(vy)
    cmz, cpz, cdz = axis(vz)
    diag = cdx + cdy + cdz
    # ghost cells: u_ghost = -u_i  ->  diag -= coupling of the missing neighbour
    diag = diag - np.where(x == 0, cmx, 0) - np.where(x == N - 1, cpx, 0)
    diag = diag - np.where(y == 0, cmy, 0) - np.where(y == N - 1, cpy, 0)
    diag = diag - np.where(z == 0, cmz, 0) - np.where(z == N - 1, cpz, 0)
    cols = np.stack([idx - N * N, idx - N, idx - 1, idx, idx + 1, idx + N, idx + N * N], axis=1)
    mask = np.stack([z > 0, y > 0, x > 0, np.ones(n, bool), x < N - 1, y < N - 1, z < N - 1], axis=1)
    vals = np.stack([cmz, cmy, cmx, diag, cpx, cpy, cpz], axis=1)
    A = _from_slots(n, cols, vals, mask)
    rng = np.random.default_rng(seed)
    b = A.matvec(np.ones(n)) + 0.01 * rng.standard_normal(n)
    peclet = float(np.max(np.abs(np.stack([vx, vy, vz]))) * h / 2.0)
    return A, b, peclet


def grf2d(N: int, corr: float, rng) -> np.ndarray:
    """Gaussian random field on a periodic N x N grid: white noise (one
    rng.standard_normal((N, N)) draw) convolved with exp(-r^2 / (2 corr^2)) by
    FFT, scaled to zero mean and unit variance."""
    w = rng.standard_normal((N, N))
    d = np.minimum(np.arange(N), N - np.arange(N)).astype(np.float64)
    ker = np.exp(-(d[:, None] ** 2 + d[None, :] ** 2) / (2.0 * corr * corr))
    g = np.real(np.fft.ifft2(np.fft.fft2(w) * np.fft.fft2(ker)))
    g -= g.mean()
    return g / g.std()


def aniso2d_grf(N: int = 512, seed: int = 4, corr: float = 16.0, ratio: float = 10.0, nrhs: int = 32):
    """2D anisotropic diffusion on N x N cells (the differentiable-solve workload).

    kappa = exp(GRF) with correlation length `corr` cells (grf2d, first draw of
    default_rng(seed)); face coefficients are harmonic means of the two cells'
    kappa, times `ratio` on x-faces (kappa_x = ratio kappa_y).  Dirichlet
    boundary faces use the boundary cell's kappa (times ratio on x).
    A = sum_f k_f (e_i - e_j)(e_i - e_j)^T + sum_boundary k_f e_i e_i^T (SPD).
    Then B ~ N(0,1) (nrhs, n) and X_target ~ N(0,1) (nrhs, n), in that order.
    Returns (A, B, X_target, kappa)."""
    rng = np.random.default_rng(seed)
    kap = np.exp(grf2d(N, corr, rng))          # kap[y, x]
    kx = np.empty((N, N + 1))
    ky = np.empty((N + 1, N))
    kx[:, 1:N] = ratio * 2.0 * kap[:, :-1] * kap[:, 1:] / (kap[:, :-1] + kap[:, 1:])
    ky[1:N, :] = 2.0 * kap[:-1, :] * kap[1:, :] / (kap[:-1, :] + kap[1:, :])
    kx[:, 0], kx[:, N] = ratio * kap[:, 0], ratio * kap[:, N - 1]
    ky[0, :], ky[N, :] = kap[0, :], kap[N - 1, :]
    n = N * N
    diag = (kx[:, :N] + kx[:, 1:] + ky[:N, :] + ky[1:, :]).reshape(n)
    idx = np.arange(n, dtype=np.int64)
    x, y = idx % N, idx // N
    cols = np.stack([idx - N, idx - 1, idx, idx + 1, idx + N], axis=1)
    mask = np.stack([y > 0, x > 0, np.ones(n, bool), x < N - 1, y < N - 1], axis=1)
    vals = np.stack([-ky[:N, :].reshape(n), -kx[:, :N].reshape(n), diag, -kx[:, 1:].reshape(n),
                     -ky[1:, :].reshape(n)], axis=1)
    A = _from_slots(n, cols, vals, mask)
    B = rng.standard_normal((nrhs, n))
    Xt = rng.standard_normal((nrhs, n))
    return A, B, Xt, kap


def _edge_stencil(shape, dirs, rng, sigma: float) -> CSR:
    """SPD stencil matrix on a grid of `shape` (x fastest) from per-edge
    coefficients: for every positive direction d in `dirs` and every cell p of
    the grid padded by one ghost layer, one draw k = exp(sigma N(0,1)) for the
    edge (p, p + d).  An edge between two cells adds k (e_i - e_j)(e_i - e_j)^T;
    an edge from a cell to a ghost (Dirichlet boundary) adds k to the cell's
    diagonal; ghost-ghost edges are dropped."""
    dim = len(shape)
    pad = tuple(s + 2 for s in shape[::-1])          # padded grid, slowest axis first
    n = int(np.prod(shape))
    grids = np.meshgrid(*[np.arange(-1, s + 1) for s in shape[::-1]], indexing="ij")
    coords = [g.ravel() for g in grids[::-1]]       # x, y (, z) of every padded cell

    def linear(c):
        lin = np.zeros(c[0].size, np.int64)
        stride = 1
        for a in range(dim):
            lin += np.clip(c[a], 0, shape[a] - 1) * stride
            stride *= shape[a]
        return lin

    def inside_of(c):
        ok = np.ones(c[0].size, bool)
        for a in range(dim):
            ok &= (c[a] >= 0) & (c[a] < shape[a])
        return ok

    inside, lin = inside_of(coords), linear(coords)
    diag = np.zeros(n)
    rows, cols, vals = [], [], []
    for d in dirs:
        k = np.exp(sigma * rng.standard_normal(pad)).ravel()
        q = [coords[a] + d[a] for a in range(dim)]
        inpad = np.ones(inside.size, bool)
        for a in range(dim):
            inpad &= (q[a] >= -1) & (q[a] <= shape[a])
        qin, ql = inside_of(q), linear(q)
        both = inside & qin & inpad
        np.add.at(diag, lin[both], k[both])
        np.add.at(diag, ql[both], k[both])
        rows += [lin[both], ql[both]]
        cols += [ql[both], lin[both]]
        vals += [-k[both], -k[both]]
        one = inpad & (inside ^ qin)                  # cell - ghost: boundary term of the inside cell
        np.add.at(diag, np.where(inside, lin, ql)[one], k[one])
    rows.append(np.arange(n))
    cols.append(np.arange(n))
    vals.append(diag)
    import scipy.sparse as sp
    S = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    S.sort_indices()
    return CSR(n, S.indptr.astype(np.int32), S.indices.astype(np.int32), S.data.astype(np.float64))


def batch_specs(nsys: int = 512, seed: int = 3, side2d=(32, 512), side3d=(16, 64), rhs=(1, 16)):
    """The batched workload's system list without building it: for every system
    (kind, side, nrhs, n, nnz), drawn exactly as batch_systems draws them.  A 2D
    5-point system has n = side^2 and nnz = 5 n - 4 side; a 3D 27-point system
    has n = side^3 and nnz = (3 side - 2)^3 (each axis couples a cell to itself
    and its two neighbours: 3 side - 2 pairs per axis)."""
    meta = np.random.default_rng(seed)
    out = []
    for _ in range(nsys):
        kind = "3d27" if meta.random() < 0.5 else "2d5"
        lo, hi = side3d if kind == "3d27" else side2d
        side = int(meta.integers(lo, hi + 1))
        nr = int(meta.integers(rhs[0], rhs[1] + 1))
        if kind == "2d5":
            n, nnz = side * side, 5 * side * side - 4 * side
        else:
            n, nnz = side ** 3, (3 * side - 2) ** 3
        out.append((kind, side, nr, n, nnz))
    return out


def batch_systems(nsys: int = 512, seed: int = 3, side2d=(32, 512), side3d=(16, 64), rhs=(1, 16),
                  sigma: float = 0.5, only=None):
    """The batched workload: nsys independent SPD systems of uneven size.

    default_rng(seed) first draws, for every system in order, its kind (2D
    5-point or 3D 27-point, probability 1/2 each), its side (uniform integer in
    side2d / side3d, inclusive) and its number of right-hand sides (uniform in
    rhs, inclusive).  System k then uses its own stream
    SeedSequence(seed).spawn(nsys)[k]: edge coefficients exp(sigma N(0,1))
    (sigma the standard deviation) via _edge_stencil, then its right-hand sides
    ~ N(0,1).  Returns a list of (kind, side, A, B) with B of shape (nrhs, n);
    with `only` (system indices) just those systems, in that order, identical
    to the same entries of the full list."""
    specs = batch_specs(nsys, seed, side2d, side3d, rhs)
    seeds = np.random.SeedSequence(seed).spawn(nsys)
    dirs2 = [(1, 0), (0, 1)]
    dirs3 = [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)
             if (dz, dy, dx) > (0, 0, 0)]                                  # 13 of the 26 neighbours
    out = []
    for k in (range(nsys) if only is None else only):
        kind, side, nr, _, _ = specs[k]
        rng = np.random.default_rng(seeds[k])
        if kind == "2d5":
            A = _edge_stencil((side, side), dirs2, rng, sigma)
        else:
            A = _edge_stencil((side, side, side), dirs3, rng, sigma)
        out.append((kind, side, A, rng.standard_normal((nr, A.n))))
    return out


def random_csr(n: int, ncols: int, density: float, seed: int, shuffle_cols: bool = True,
               empty_rows: float = 0.0, dense_tile_rows: int = 0) -> CSR:
    """Random CSR with unsorted columns (when shuffle_cols), optional empty rows
    and optional fully dense 16x16 tiles (256 entries: exercises the uint8
    end-offset wrap of the reference's row lists)."""
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(n):
        if rng.random() < empty_rows:
            rows.append(np.zeros(0, dtype=np.int64))
            continue
        k = max(1, rng.binomial(ncols, density))
        rows.append(rng.choice(ncols, size=min(k, ncols), replace=False))
    for t in range(dense_tile_rows):
        R = rng.integers(0, n // 16)
        J = rng.integers(0, ncols // 16)
        for r in range(16):
            i = R * 16 + r
            rows[i] = np.union1d(rows[i], np.arange(J * 16, J * 16 + 16))
    cols, ptr = [], [0]
    for r in rows:
        r = np.asarray(r, dtype=np.int64)
        r = rng.permutation(r) if shuffle_cols else np.sort(r)
        cols.append(r)
        ptr.append(ptr[-1] + r.size)
    colidx = np.concatenate(cols) if cols else np.zeros(0, dtype=np.int64)
    val = rng.standard_normal(colidx.size)
    return CSR(n, np.asarray(ptr, dtype=np.int32), colidx.astype(np.int32), val)


def write_cbd(path: str, A: CSR, ncols: int | None = None) -> None:
    """Binary CSR: int32 rows, int32 cols, int64 nnz, int64 rowptr[rows+1],
    int32 colidx[nnz], float64 val[nnz] (the .cbd layout of biio.h:74-97)."""
    with open(path, "wb") as f:
        np.array([A.n, ncols if ncols is not None else A.n], dtype=np.int32).tofile(f)
        np.array([A.nnz], dtype=np.int64).tofile(f)
        A.rowptr.astype(np.int64).tofile(f)
        A.colidx.astype(np.int32).tofile(f)
        A.val.astype(np.float64).tofile(f)


def write_mtx(path: str, A: CSR, ncols: int | None = None, symmetric: bool = False,
              field: str = "real") -> None:
    """Matrix Market coordinate file (1-based), entries in CSR order."""
    rows = np.repeat(np.arange(A.n), np.diff(A.rowptr))
    cols = A.colidx
    vals = A.val
    if symmetric:
        keep = cols <= rows
        rows, cols, vals = rows[keep], cols[keep], vals[keep]
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {field} {'symmetric' if symmetric else 'general'}\n")
        f.write("% generated\n")
        f.write(f"{A.n} {ncols if ncols is not None else A.n} {rows.size}\n")
        if field == "pattern":
            for r, c in zip(rows, cols):
                f.write(f"{r + 1} {c + 1}\n")
        elif field == "integer":
            for r, c, v in zip(rows, cols, vals):
                f.write(f"{r + 1} {c + 1} {int(v)}\n")
        else:
            for r, c, v in zip(rows, cols, vals):
                f.write(f"{r + 1} {c + 1} {v:.17g}\n")
