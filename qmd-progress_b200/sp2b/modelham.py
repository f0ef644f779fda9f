"""Seeded model Hamiltonians for the SP2 workloads, plus a MatrixMarket reader.

The reference builds its model Hamiltonians in ``src/prg_modelham_mod.F90``
(``prg_twolevel_model``, :116-202, a two-level chain with exponentially decaying
hopping).  The generators below follow the same pattern with the parameters of
the benchmark workloads:

* ``two_band_1d``   - two-band periodic chain: onsite -1 / +1 (even / odd site) plus
  N(0, 0.05^2) noise, hopping -0.2 exp(-(d-1)) for periodic distance 1 <= d <= 4.
* ``cubic_3d``      - L^3 simple-cubic periodic lattice, one orbital per site, onsite
  U[-1, 1] + 0.8 (-1)^(x+y+z), hopping -0.25 exp(-(r-1)) for r <= 2 (offsets with
  r in {1, sqrt 2, sqrt 3, 2}); returned sparse (CSR) or dense.
* ``random_symmetric`` - A_ij ~ N(0,1)/sqrt(N), symmetrised (the adjoint's weight matrix).

All return FP64 numpy arrays in the row-major layout the library expects (the
matrices are symmetric, so row- and column-major coincide).
"""
from __future__ import annotations

import math

import numpy as np


def two_band_1d(n: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    h = np.zeros((n, n), dtype=np.float64)
    onsite = np.where(np.arange(n) % 2 == 0, -1.0, 1.0) + rng.normal(0.0, 0.05, n)
    h[np.arange(n), np.arange(n)] = onsite
    i = np.arange(n)
    for d in range(1, 5):
        if 2 * d > n and d != n - d:
            # for tiny rings each pair is reached once, at its shortest distance
            pass
        t = -0.2 * math.exp(-(d - 1))
        j = (i + d) % n
        dist = np.minimum(np.abs(i - j), n - np.abs(i - j))
        mask = (dist == d) & (i != j)
        h[i[mask], j[mask]] = t
        h[j[mask], i[mask]] = t
    return h


def _cubic_offsets():
    offs = []
    for dx in range(-2, 3):
        for dy in range(-2, 3):
            for dz in range(-2, 3):
                r2 = dx * dx + dy * dy + dz * dz
                if 0 < r2 <= 4:
                    offs.append((dx, dy, dz, math.sqrt(r2)))
    return offs


def cubic_3d_csr(L: int = 32, seed: int = 0, threshold: float = 1e-5):
    """3D lattice Hamiltonian as CSR (row_ptr int64, col int32, val float64), N = L^3.

    Site index s = x + L*(y + L*z).  Elements with |h| <= threshold are dropped.
    """
    rng = np.random.default_rng(seed)
    n = L ** 3
    s = np.arange(n)
    x = s % L
    y = (s // L) % L
    z = s // (L * L)
    onsite = rng.uniform(-1.0, 1.0, n) + 0.8 * np.where((x + y + z) % 2 == 0, 1.0, -1.0)
    rows = [s]
    cols = [s]
    vals = [onsite]
    for dx, dy, dz, r in _cubic_offsets():
        t = -0.25 * math.exp(-(r - 1.0))
        if abs(t) <= threshold:
            continue
        nb = ((x + dx) % L) + L * (((y + dy) % L) + L * ((z + dz) % L))
        rows.append(s)
        cols.append(nb)
        vals.append(np.full(n, t))
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = np.concatenate(vals)
    # For L <= 4 periodic images coincide; sum duplicates.
    key = r * n + c
    order = np.argsort(key, kind="stable")
    key, v = key[order], v[order]
    uniq, start = np.unique(key, return_index=True)
    v = np.add.reduceat(v, start)
    r = (uniq // n).astype(np.int64)
    c = (uniq % n).astype(np.int32)
    keep = np.abs(v) > threshold
    r, c, v = r[keep], c[keep], v[keep]
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(row_ptr, r + 1, 1)
    row_ptr = np.cumsum(row_ptr)
    return row_ptr, c, v


def csr_to_dense(row_ptr, col, val, n):
    h = np.zeros((n, n), dtype=np.float64)
    for i in range(n):
        a, b = row_ptr[i], row_ptr[i + 1]
        h[i, col[a:b]] = val[a:b]
    return h


def cubic_3d(L: int = 32, seed: int = 0, threshold: float = 1e-5) -> np.ndarray:
    rp, c, v = cubic_3d_csr(L, seed, threshold)
    return csr_to_dense(rp, c, v, L ** 3)


def random_symmetric(n: int, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    g = rng.normal(0.0, 1.0, (n, n)) / math.sqrt(n)
    return (g + g.T) / math.sqrt(2.0)


def read_mtx(path: str) -> np.ndarray:
    """Dense FP64 matrix from a MatrixMarket ``coordinate real general|symmetric`` file."""
    with open(path) as f:
        header = f.readline()
        symmetric = "symmetric" in header.lower()
        line = f.readline()
        while line.startswith("%"):
            line = f.readline()
        nr, nc, nnz = (int(t) for t in line.split())
        data = np.loadtxt(f, ndmin=2)
    h = np.zeros((nr, nc), dtype=np.float64)
    i = data[:, 0].astype(np.int64) - 1
    j = data[:, 1].astype(np.int64) - 1
    h[i, j] = data[:, 2]
    if symmetric:
        h[j, i] = data[:, 2]
    return h
