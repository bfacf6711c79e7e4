"""Seeded synthetic sparse matrices for the CB-SpMV workloads.

Every generator returns a :class:`Coo` whose entries are sorted by (row, col)
without duplicates -- the order the reference's Matrix Market reader hands to
``coo2block_gather`` (cb-spmv-dcu/src/io/mmio_highlevel.h:392-398), which the
CB builder needs because blocks of one block row must be contiguous.

Workloads (sizes as named by the benchmark configurations):

* ``laplacian_2d``  -- 5-point Laplacian, 256x256 grid: n=65,536, 326,656 nnz,
  diagonal 4, off-diagonals -1.
* ``power_law``     -- n=2^20, row lengths from a power law with exponent 2.1,
  lengths in [1, 20000] and a target mean; 70% of columns within +-4096 of the
  diagonal, 30% uniform; values N(0,1).
* ``stencil_27pt``  -- 64^3 grid x 3 dof, 27-point stencil with dense 3x3
  nodal couplings: n=786,432, 61,731,000 nnz (boundary-truncated).
* ``batch_uneven``  -- 512 independent matrices of uneven size and kind.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Coo:
    m: int
    n: int
    row: np.ndarray  # int32, sorted
    col: np.ndarray  # int32
    val: np.ndarray  # float64

    @property
    def nnz(self) -> int:
        return int(self.row.shape[0])


def _sorted_unique(key: np.ndarray) -> np.ndarray:
    """Sorted distinct values (np.unique without its slow hash pass)."""
    key = np.sort(key)
    if key.shape[0] == 0:
        return key
    keep = np.empty(key.shape[0], dtype=bool)
    keep[0] = True
    np.not_equal(key[1:], key[:-1], out=keep[1:])
    return key[keep]


def _finish(m: int, n: int, row, col, val) -> Coo:
    return Coo(m, n, np.ascontiguousarray(row, dtype=np.int32),
               np.ascontiguousarray(col, dtype=np.int32),
               np.ascontiguousarray(val, dtype=np.float64))


def laplacian_2d(nx: int = 256, ny: int = 256) -> Coo:
    """5-point Laplacian on an nx-by-ny grid, natural ordering."""
    n = nx * ny
    i = np.arange(n, dtype=np.int64)
    x = i % nx
    y = i // nx
    # candidate columns in ascending order: i-nx, i-1, i, i+1, i+nx
    cols = np.stack([i - nx, i - 1, i, i + 1, i + nx], axis=1)
    ok = np.stack([y > 0, x > 0, np.ones(n, bool), x < nx - 1, y < ny - 1],
                  axis=1)
    vals = np.where(np.arange(5) == 2, 4.0, -1.0)[None, :].repeat(n, 0)
    rows = np.repeat(i, 5).reshape(n, 5)
    return _finish(n, n, rows[ok], cols[ok], vals[ok])


def _zipf_mandelbrot_offset(alpha: float, kmax: int, mean: float) -> float:
    """Offset k0 of p(k) ~ (k + k0)^-alpha on k in [1, kmax] giving ``mean``.

    A plain discrete power law with minimum 1 and exponent 2.1 has a mean near
    6.3 at kmax=20000; shifting it keeps the minimum at 1 and the tail
    exponent at alpha while moving the mean to the requested value.
    """
    k = np.arange(1, kmax + 1, dtype=np.float64)

    def mean_of(k0):
        w = (k + k0) ** (-alpha)
        return float((w * k).sum() / w.sum())

    lo, hi = -0.99, 1000.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if mean_of(mid) < mean:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def power_law_lengths(rng, n: int, alpha: float, kmin: int, kmax: int,
                      mean: float) -> np.ndarray:
    k0 = _zipf_mandelbrot_offset(alpha, kmax, mean)
    k = np.arange(1, kmax + 1, dtype=np.float64)
    w = (k + k0) ** (-alpha)
    cdf = np.cumsum(w / w.sum())
    lengths = np.searchsorted(cdf, rng.random(n), side="right") + 1
    return np.clip(lengths, kmin, kmax).astype(np.int64)


def power_law(n: int = 1 << 20, seed: int = 1, alpha: float = 2.1,
              kmin: int = 1, kmax: int = 20000, mean: float = 16.0,
              local_frac: float = 0.7, band: int = 4096,
              mean_boost: float = 1.065) -> Coo:
    """Power-law row lengths, 70% near-diagonal columns, N(0,1) values.

    Duplicate (row, col) draws are removed, so the realised mean is slightly
    below the drawn mean; ``mean_boost`` scales the drawn mean to compensate.
    """
    rng = np.random.default_rng(seed)
    lengths = power_law_lengths(rng, n, alpha, kmin, min(kmax, n),
                                mean * mean_boost)
    total = int(lengths.sum())
    rows = np.repeat(np.arange(n, dtype=np.int64), lengths)
    local = rng.random(total) < local_frac
    lo = np.maximum(rows - band, 0)
    hi = np.minimum(rows + band, n - 1)
    near = lo + np.floor(rng.random(total) * (hi - lo + 1)).astype(np.int64)
    far = rng.integers(0, n, size=total, dtype=np.int64)
    cols = np.where(local, near, far)
    key = _sorted_unique(rows * n + cols)
    rows = key // n
    cols = key % n
    vals = rng.standard_normal(key.shape[0])
    return _finish(n, n, rows, cols, vals)


def stencil_27pt(g: int = 64, dof: int = 3, seed: int = 2) -> Coo:
    """27-point stencil on a g^3 grid with dense dof x dof nodal couplings.

    Off-diagonal values U[-1,1]; each diagonal entry is 1 + the row's sum of
    off-diagonal magnitudes (strict diagonal dominance).
    """
    rng = np.random.default_rng(seed)
    nodes = g ** 3
    n = nodes * dof
    node = np.arange(nodes, dtype=np.int64)
    x, y, z = node % g, (node // g) % g, node // (g * g)
    nbrs, oks = [], []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                ok = ((x + dx >= 0) & (x + dx < g) & (y + dy >= 0)
                      & (y + dy < g) & (z + dz >= 0) & (z + dz < g))
                nbrs.append(node + dx + g * dy + g * g * dz)
                oks.append(ok)
    nbr = np.stack(nbrs, axis=1)          # nodes x 27, ascending per node
    ok = np.stack(oks, axis=1)
    counts = ok.sum(axis=1)               # valid neighbours per node
    nbr_flat = nbr[ok]                    # row-major: node, then neighbour
    node_start = np.concatenate([[0], np.cumsum(counts)])
    # row (node, d) lists, for each valid neighbour, its dof columns
    row_len = counts * dof                # per node, same for every d
    rows = np.repeat(np.arange(n, dtype=np.int64), np.repeat(row_len, dof))
    # build columns per node block then tile over d
    per_node_cols = (nbr_flat[:, None] * dof
                     + np.arange(dof)[None, :]).reshape(-1)  # node-major
    pos = np.repeat(node_start[:-1] * dof, counts * dof * dof)
    within = np.arange(rows.shape[0], dtype=np.int64)
    row_start = np.concatenate([[0], np.cumsum(np.repeat(row_len, dof))])
    within = within - np.repeat(row_start[:-1], np.repeat(row_len, dof))
    cols = per_node_cols[pos + within]
    vals = rng.uniform(-1.0, 1.0, size=rows.shape[0])
    diag = rows == cols
    offabs = np.bincount(rows, weights=np.where(diag, 0.0, np.abs(vals)),
                         minlength=n)
    vals[diag] = 1.0 + offabs[rows[diag]]
    return _finish(n, n, rows, cols, vals)


def uniform_random(rng, n: int, density: float, cap: int = 64) -> Coo:
    lengths = np.minimum(rng.binomial(n, density, size=n), cap)
    lengths = np.maximum(lengths, 1)
    total = int(lengths.sum())
    rows = np.repeat(np.arange(n, dtype=np.int64), lengths)
    cols = rng.integers(0, n, size=total, dtype=np.int64)
    key = _sorted_unique(rows * n + cols)
    vals = rng.standard_normal(key.shape[0])
    return _finish(n, n, key // n, key % n, vals)


def banded(rng, n: int, bw: int) -> Coo:
    """All entries with |i - j| <= bw."""
    i = np.arange(n, dtype=np.int64)
    off = np.arange(-bw, bw + 1, dtype=np.int64)
    cols = i[:, None] + off[None, :]
    ok = (cols >= 0) & (cols < n)
    rows = np.repeat(i, off.shape[0]).reshape(n, -1)
    vals = rng.standard_normal(int(ok.sum()))
    return _finish(n, n, rows[ok], cols[ok], vals)


@dataclasses.dataclass
class BatchItem:
    kind: str
    coo: Coo
    nrhs: int


def batch_uneven(count: int = 512, seed: int = 4, nmin: int = 1024,
                 nmax: int = 131072) -> list:
    """Uneven batch: n log-uniform in [nmin, nmax]; banded (bandwidth 1-64),
    power-law (alpha 2.1) or uniform random (density 1e-4..1e-2, <= 64 per
    row); 1-16 right-hand sides each."""
    rng = np.random.default_rng(seed)
    items = []
    for _ in range(count):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        kind = ("banded", "power_law", "uniform")[int(rng.integers(0, 3))]
        nrhs = int(rng.integers(1, 17))
        if kind == "banded":
            coo = banded(rng, n, int(rng.integers(1, 65)))
        elif kind == "power_law":
            coo = power_law(n, seed=int(rng.integers(0, 2**31)),
                            band=max(16, n // 256), kmax=min(20000, n))
        else:
            density = math.exp(rng.uniform(math.log(1e-4), math.log(1e-2)))
            coo = uniform_random(rng, n, density)
        items.append(BatchItem(kind, coo, nrhs))
    return items


def random_small(rng, m: int, n: int, nnz: int, dup: bool = False,
                 unit: bool = False) -> Coo:
    """Small random COO for exhaustive tests; optionally with duplicates
    (kept, as the reference builder sums them) and unit values."""
    rows = rng.integers(0, m, size=nnz, dtype=np.int64)
    cols = rng.integers(0, n, size=nnz, dtype=np.int64)
    if not dup:
        key = _sorted_unique(rows * n + cols)
        rows, cols = key // n, key % n
    else:
        order = np.argsort(rows, kind="stable")
        rows, cols = rows[order], cols[order]
    vals = (np.ones(rows.shape[0]) if unit
            else rng.standard_normal(rows.shape[0]))
    return _finish(m, n, rows, cols, vals)


def uniform_x(n: int, seed: int, nrhs: int = 1, lo=-1.0, hi=1.0) -> np.ndarray:
    """x ~ U[lo, hi] from ``seed`` (column-major n x nrhs when nrhs > 1)."""
    rng = np.random.default_rng(seed)
    x = rng.uniform(lo, hi, size=(nrhs, n))
    return x[0].copy() if nrhs == 1 else np.ascontiguousarray(x)
