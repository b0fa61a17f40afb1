"""Seeded synthetic systems for the solver path (numpy, host side).

These reproduce the shapes, sizes and value distributions of the reference's
generators (2D/3D stencils in iterative/BiCGSTAB/benchmark.py:58-108 and
iterative/cgd/comp_bench.py, diagonally dominant block matrices in
iterative/BiCGSTAB/benchmark.py:29-56) at the sizes this package is measured
on.  All randomness comes from ``numpy.random.default_rng(seed)``.

Conventions
-----------
* Cell (i, j[, k]) of an nx x ny[ x nz] grid is row ``i + nx*(j + ny*k)``.
* Variable-coefficient operators use face conductivity = geometric mean of the
  two cell conductivities, ``k_f = sqrt(k_a k_b)``; a Dirichlet boundary face
  adds the cell's own conductivity to the diagonal.
* Gaussian random fields: white noise filtered by a Gaussian kernel whose
  standard deviation is the correlation length (in cells), then scaled to
  zero mean and standard deviation ``sigma``.
* Matrix values are rounded to FP32: the FP32 values define the system.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class Coo:
    rows: np.ndarray      # int64
    cols: np.ndarray      # int64
    vals: np.ndarray      # float32
    n: int

    @property
    def nnz(self) -> int:
        return int(self.rows.shape[0])

    def keys(self) -> np.ndarray:
        """Packed int64 keys (row << 32) | col, as pack_keys builds them
        (iterative/BiCGSTAB/benchmark.py:110-114)."""
        return (self.rows.astype(np.int64) << 32) | self.cols.astype(np.int64)

    def shuffled(self, seed: int) -> "Coo":
        p = np.random.default_rng(seed).permutation(self.nnz)
        return Coo(self.rows[p], self.cols[p], self.vals[p], self.n)

    def to_csr(self):
        """Stable (row, col) order CSR arrays: (row_ptr, col_ind, vals)."""
        order = np.lexsort((self.cols, self.rows))
        rp = np.zeros(self.n + 1, np.int64)
        np.add.at(rp, self.rows + 1, 1)
        return (np.cumsum(rp).astype(np.int32), self.cols[order].astype(np.int32),
                self.vals[order].astype(np.float32))


def _assemble(n, diag, pairs):
    """diag: float64[n]; pairs: list of (a, b, k) arrays for symmetric -k."""
    rows = [np.arange(n, dtype=np.int64)]
    cols = [np.arange(n, dtype=np.int64)]
    vals = [diag]
    for a, b, k in pairs:
        rows += [a, b]
        cols += [b, a]
        vals += [-k, -k]
    return Coo(np.concatenate(rows), np.concatenate(cols),
               np.concatenate(vals).astype(np.float32), n)


def laplacian_2d(nx: int, ny: int | None = None) -> Coo:
    """5-point Laplacian, Dirichlet: diagonal 4, off-diagonals -1."""
    ny = nx if ny is None else ny
    n = nx * ny
    idx = np.arange(n, dtype=np.int64).reshape(ny, nx)
    e = idx[:, :-1].ravel(), idx[:, 1:].ravel()
    s = idx[:-1, :].ravel(), idx[1:, :].ravel()
    one = lambda a: np.ones(a[0].shape[0])
    return _assemble(n, np.full(n, 4.0), [(e[0], e[1], one(e)), (s[0], s[1], one(s))])


def gaussian_field(shape, sigma: float, corr_len: float, seed: int) -> np.ndarray:
    """Gaussian random field by FFT filtering of white noise (float64)."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    fw = np.fft.rfftn(w)
    freqs = [np.fft.fftfreq(s) for s in shape[:-1]] + [np.fft.rfftfreq(shape[-1])]
    k2 = np.zeros(fw.shape)
    for ax, f in enumerate(freqs):
        sh = [1] * len(shape)
        sh[ax] = f.shape[0]
        k2 = k2 + (2 * np.pi * f.reshape(sh)) ** 2
    g = np.fft.irfftn(fw * np.exp(-0.5 * k2 * corr_len ** 2), s=shape, axes=tuple(range(len(shape))))
    g -= g.mean()
    sd = g.std()
    return g * (sigma / sd) if sd > 0 else g


def diffusion(kcell: np.ndarray) -> Coo:
    """Variable-coefficient diffusion on a 2D (ny, nx) or 3D (nz, ny, nx)
    conductivity array; 5- or 7-point, Dirichlet."""
    shape = kcell.shape
    n = int(np.prod(shape))
    idx = np.arange(n, dtype=np.int64).reshape(shape)
    diag = np.zeros(shape)
    pairs = []
    for ax in range(len(shape)):
        lo = [slice(None)] * len(shape)
        hi = [slice(None)] * len(shape)
        lo[ax] = slice(None, -1)
        hi[ax] = slice(1, None)
        kf = np.sqrt(kcell[tuple(lo)] * kcell[tuple(hi)])
        diag[tuple(lo)] += kf
        diag[tuple(hi)] += kf
        pairs.append((idx[tuple(lo)].ravel(), idx[tuple(hi)].ravel(), kf.ravel()))
        first = [slice(None)] * len(shape)
        last = [slice(None)] * len(shape)
        first[ax] = 0
        last[ax] = -1
        diag[tuple(first)] += kcell[tuple(first)]
        diag[tuple(last)] += kcell[tuple(last)]
    return _assemble(n, diag.ravel(), pairs)


def lognormal_diffusion_2d(nx, ny, sigma, corr_len, seed) -> Coo:
    return diffusion(np.exp(gaussian_field((ny, nx), sigma, corr_len, seed)))


def lognormal_diffusion_3d(m, sigma, corr_len, seed) -> Coo:
    return diffusion(np.exp(gaussian_field((m, m, m), sigma, corr_len, seed)))


def graph_laplacian(n: int, mean_degree: float, seed: int, shift: float = 1e-2) -> Coo:
    """Random graph Laplacian: n*deg/2 uniform random edges (deduplicated, no
    self loops), weights U(0.1, 1), plus shift*I."""
    rng = np.random.default_rng(seed)
    m = int(round(n * mean_degree / 2))
    a = rng.integers(0, n, m)
    b = rng.integers(0, n - 1, m)
    b = np.where(b >= a, b + 1, b)
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = np.unique(lo * n + hi)
    lo, hi = key // n, key % n
    w = rng.uniform(0.1, 1.0, key.shape[0])
    diag = np.full(n, shift)
    np.add.at(diag, lo, w)
    np.add.at(diag, hi, w)
    return _assemble(n, diag, [(lo, hi, w)])


@dataclass
class Bcsr:
    row_ptr: np.ndarray   # int32[nbr+1]
    col_ind: np.ndarray   # int32[nblocks]
    vals: np.ndarray      # float32[nblocks*B*B], row-major blocks
    block: int
    n: int

    def to_coo(self, drop_zeros: bool = True) -> Coo:
        B = self.block
        nb = self.col_ind.shape[0]
        br = np.repeat(np.arange(self.row_ptr.shape[0] - 1), np.diff(self.row_ptr))
        r = (br[:, None, None] * B + np.arange(B)[None, :, None]) + 0 * np.arange(B)[None, None, :]
        c = (self.col_ind[:, None, None].astype(np.int64) * B + np.arange(B)[None, None, :]) \
            + 0 * np.arange(B)[None, :, None]
        v = self.vals.reshape(nb, B, B)
        r, c, v = r.ravel().astype(np.int64), c.ravel(), v.ravel()
        if drop_zeros:
            keep = v != 0
            r, c, v = r[keep], c[keep], v[keep]
        return Coo(r, c, v.astype(np.float32), self.n)


def block_dominant(n_block_rows: int, off_blocks: int, seed: int, block: int = 4) -> Bcsr:
    """Nonsymmetric diagonally dominant BCSR: per block row a diagonal block
    plus ``off_blocks`` off-diagonal blocks at distinct block columns drawn
    uniformly without replacement; off-diagonal entries U(-1, 1); diagonal
    block = I * (row abs-sum + 1)."""
    rng = np.random.default_rng(seed)
    nbr, B, k = n_block_rows, block, off_blocks
    draws = 3 * k
    cand = rng.integers(0, nbr - 1, (nbr, draws))
    cand = np.where(cand >= np.arange(nbr)[:, None], cand + 1, cand)
    order = np.argsort(cand, axis=1, kind="stable")
    srt = np.take_along_axis(cand, order, axis=1)
    dup_sorted = np.zeros_like(srt, dtype=bool)
    dup_sorted[:, 1:] = srt[:, 1:] == srt[:, :-1]
    dup = np.zeros_like(dup_sorted)
    np.put_along_axis(dup, order, dup_sorted, axis=1)
    ok = ~dup
    take = ok & (np.cumsum(ok, axis=1) <= k)
    assert (take.sum(1) == k).all(), "not enough distinct block columns drawn"
    offc = cand[take].reshape(nbr, k)
    offv = rng.uniform(-1.0, 1.0, (nbr, k, B, B)).astype(np.float32)
    rowsum = np.abs(offv.astype(np.float64)).sum(axis=(1, 3))        # (nbr, B)
    diagv = np.zeros((nbr, 1, B, B), np.float32)
    diagv[:, 0, np.arange(B), np.arange(B)] = (rowsum + 1.0).astype(np.float32)
    cols = np.concatenate([np.arange(nbr)[:, None], offc], axis=1)
    vals = np.concatenate([diagv, offv], axis=1)
    o = np.argsort(cols, axis=1, kind="stable")
    cols = np.take_along_axis(cols, o, axis=1)
    vals = np.take_along_axis(vals, o[:, :, None, None], axis=1)
    rp = (np.arange(nbr + 1) * (k + 1)).astype(np.int32)
    return Bcsr(rp, cols.ravel().astype(np.int32), vals.ravel(), B, nbr * B)


def rhs(n: int, seed: int) -> np.ndarray:
    """b ~ N(0, 1) in FP32."""
    return np.random.default_rng(seed).standard_normal(n).astype(np.float32)


# Named configurations ------------------------------------------------------

def laplacian_256() -> Coo:
    """2D 5-point Laplacian over 256x256, n = 65,536, nnz = 326,656."""
    return laplacian_2d(256)


def block_dominant_65536(seed: int = 0) -> Bcsr:
    """65,536 block rows of 4x4 blocks, 9 blocks per row (n = 262,144)."""
    return block_dominant(65536, 8, seed)


def diffusion_256cubed(seed: int = 0) -> Coo:
    """3D 7-point log-normal diffusion, 256^3 cells, sigma 1, corr length 8."""
    return lognormal_diffusion_3d(256, 1.0, 8.0, seed)


def diffusion_512sq(seed: int) -> Coo:
    """2D 5-point log-normal diffusion, 512^2 cells, sigma 1.5, corr length 16."""
    return lognormal_diffusion_2d(512, 512, 1.5, 16.0, seed)


def lognormal_diffusion_2d_torch(nx: int, ny: int, sigma: float, corr_len: float, seed: int,
                                 device="cuda"):
    """Same operator as ``lognormal_diffusion_2d`` (same seed -> same white
    noise from numpy), with the FFT filter and the assembly done by torch on
    ``device``.  Returns (keys int64, values float32, n) tensors on ``device``."""
    import torch

    w = np.random.default_rng(seed).standard_normal((ny, nx))
    wt = torch.from_numpy(w).to(device)
    fw = torch.fft.rfftn(wt)
    fy = torch.fft.fftfreq(ny, device=device, dtype=torch.float64)
    fx = torch.fft.rfftfreq(nx, device=device, dtype=torch.float64)
    k2 = (2 * np.pi * fy)[:, None] ** 2 + (2 * np.pi * fx)[None, :] ** 2
    g = torch.fft.irfftn(fw * torch.exp(-0.5 * k2 * corr_len ** 2), s=(ny, nx))
    g = g - g.mean()
    sd = g.std(unbiased=False)
    g = g * (sigma / sd)
    k = torch.exp(g)
    n = nx * ny
    idx = torch.arange(n, device=device, dtype=torch.int64).reshape(ny, nx)
    diag = torch.zeros((ny, nx), device=device, dtype=torch.float64)
    ky = torch.sqrt(k[:-1, :] * k[1:, :])                 # faces between rows j, j+1
    diag[:-1, :] += ky
    diag[1:, :] += ky
    diag[0, :] += k[0, :]
    diag[-1, :] += k[-1, :]
    kx = torch.sqrt(k[:, :-1] * k[:, 1:])                 # faces between columns i, i+1
    diag[:, :-1] += kx
    diag[:, 1:] += kx
    diag[:, 0] += k[:, 0]
    diag[:, -1] += k[:, -1]
    a_y, b_y = idx[:-1, :].reshape(-1), idx[1:, :].reshape(-1)
    a_x, b_x = idx[:, :-1].reshape(-1), idx[:, 1:].reshape(-1)
    rows = torch.cat([idx.reshape(-1), a_y, b_y, a_x, b_x])
    cols = torch.cat([idx.reshape(-1), b_y, a_y, b_x, a_x])
    vals = torch.cat([diag.reshape(-1), -ky.reshape(-1), -ky.reshape(-1), -kx.reshape(-1),
                      -kx.reshape(-1)]).to(torch.float32)
    return (rows << 32) | cols, vals, n


def graph_laplacian_torch(n: int, mean_degree: float, seed: int, shift: float = 1e-2,
                          device="cuda"):
    """Random graph Laplacian on ``device`` (torch generator): n*deg/2 uniform
    random edges, deduplicated, no self loops, weights U(0.1, 1), plus
    shift*I.  Returns (keys, values, n)."""
    import torch

    g = torch.Generator(device=device).manual_seed(seed)
    m = int(round(n * mean_degree / 2))
    a = torch.randint(0, n, (m,), generator=g, device=device)
    b = torch.randint(0, n - 1, (m,), generator=g, device=device)
    b = torch.where(b >= a, b + 1, b)
    key = torch.unique(torch.minimum(a, b) * n + torch.maximum(a, b))
    lo, hi = key // n, key % n
    w = 0.1 + 0.9 * torch.rand(key.shape[0], generator=g, device=device, dtype=torch.float64)
    diag = torch.full((n,), shift, device=device, dtype=torch.float64)
    diag.index_add_(0, lo, w)
    diag.index_add_(0, hi, w)
    idx = torch.arange(n, device=device)
    rows = torch.cat([idx, lo, hi])
    cols = torch.cat([idx, hi, lo])
    vals = torch.cat([diag, -w, -w]).to(torch.float32)
    return (rows << 32) | cols, vals, n


def batch_plan(n_systems: int, seed: int, n_min: int = 1024, n_max: int = 65536,
               mean_degree: float = 8.0):
    """Shapes of the systems batch_systems makes, without making them:
    (kind per system: 0 grid / 1 graph, grid (nx, ny) or graph row count,
    estimated nonzeros per system) -- what a rank needs to pick its share."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_systems))
    kinds = np.arange(n_systems) % 2
    shapes, nnz = [], np.empty(n_systems, np.int64)
    for s, target in enumerate(sizes):
        if kinds[s] == 0:
            nx = max(2, int(round(np.sqrt(target))))
            ny = max(2, int(round(target / nx)))
            shapes.append((nx, ny))
            nnz[s] = 5 * nx * ny - 2 * nx - 2 * ny
        else:
            n = int(round(target))
            shapes.append(n)
            nnz[s] = int(n * (1 + mean_degree))
    return kinds.astype(np.int8), shapes, nnz


def batch_systems(n_systems: int, seed: int, n_min: int = 1024, n_max: int = 65536,
                  grid_sigma: float = 1.0, grid_corr: float = 8.0, mean_degree: float = 8.0,
                  device="cuda", select=None):
    """Independent SPD systems with row counts log-uniform in [n_min, n_max]:
    even indices are 2D 5-point log-normal diffusion grids (near-square),
    odd indices random graph Laplacians + 1e-2 I.  Returns the stacked
    (keys, values) on ``device`` with global indices, row offsets (numpy) and
    the kind of every system (0 grid, 1 graph).  ``select``: only these
    system indices, stacked in the order given (each system comes from its
    own seed, so a subset is the same systems as in the whole batch)."""
    import torch

    kinds_all, shapes, _ = batch_plan(n_systems, seed, n_min, n_max, mean_degree)
    idx = range(n_systems) if select is None else [int(i) for i in select]
    keys, vals, off, kinds = [], [], [0], []
    for s in idx:
        if kinds_all[s] == 0:
            nx, ny = shapes[s]
            k, v, n = lognormal_diffusion_2d_torch(nx, ny, grid_sigma, grid_corr,
                                                   seed * 1_000_003 + s, device)
        else:
            k, v, n = graph_laplacian_torch(shapes[s], mean_degree, seed * 1_000_003 + s,
                                            device=device)
        kinds.append(int(kinds_all[s]))
        base = off[-1]
        keys.append(k + ((base << 32) | base))
        vals.append(v)
        off.append(base + n)
    return torch.cat(keys), torch.cat(vals), np.asarray(off, np.int64), np.asarray(kinds, np.int8)


def stack(systems) -> tuple[Coo, np.ndarray]:
    """Block-diagonal stack of Coo systems: (global Coo, row offsets)."""
    off = np.zeros(len(systems) + 1, np.int64)
    off[1:] = np.cumsum([s.n for s in systems])
    rows = np.concatenate([s.rows + o for s, o in zip(systems, off)])
    cols = np.concatenate([s.cols + o for s, o in zip(systems, off)])
    vals = np.concatenate([s.vals for s in systems])
    return Coo(rows, cols, vals, int(off[-1])), off
