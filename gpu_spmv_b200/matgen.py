"""Seeded synthetic matrices for the benchmark workloads (the engine's C++ generators).

Each generator returns CSR numpy arrays ``(row uint32[n+1], col uint32[nnz],
val float64[nnz])``; the same seed gives the same matrix on any machine and thread count.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


def _take(ptr, n, dtype):
    if n == 0:
        out = np.zeros(0, dtype)
    else:
        out = np.ctypeslib.as_array(ptr, shape=(n,)).copy().view(dtype)
    L.lib().gs_free_host(C.cast(ptr, C.c_void_p))
    return out


def _finish(row, col, val, n, nnz):
    return (_take(row, n + 1, np.uint32), _take(col, nnz, np.uint32),
            _take(val, nnz, np.float64))


def laplacian2d(grid: int = 512):
    """5-point Laplacian of a grid x grid mesh (diagonal 4, off-diagonals -1)."""
    row, col, val = L.UINp(), L.UINp(), L.FPTp()
    n, nnz = L.UIN(), L.UIN()
    L.check(L.lib().gs_gen_laplacian2d(grid, C.byref(row), C.byref(col), C.byref(val),
                                       C.byref(n), C.byref(nnz)), "gs_gen_laplacian2d")
    return _finish(row, col, val, n.value, nnz.value)


def powerlaw(nrows: int = 4194304, nnz: int = 67108864, mu: float = 2.5, sigma: float = 1.2,
             max_len: int = 10000, seed: int = 1):
    """lognormal(mu, sigma) row lengths clipped to [1, max_len] and rescaled to exactly
    ``nnz``; columns uniform without replacement (sorted per row); values N(0,1)."""
    row, col, val = L.UINp(), L.UINp(), L.FPTp()
    got = L.UIN()
    L.check(L.lib().gs_gen_powerlaw(nrows, nnz, mu, sigma, max_len, seed, C.byref(row),
                                    C.byref(col), C.byref(val), C.byref(got)),
            "gs_gen_powerlaw")
    return _finish(row, col, val, nrows, got.value)


def stencil27(grid: int = 160, seed: int = 2):
    """27-point stencil on grid^3: diagonal 26, off-diagonals -1 + U(-0.1, 0.1)."""
    row, col, val = L.UINp(), L.UINp(), L.FPTp()
    n, nnz = L.UIN(), L.UIN()
    L.check(L.lib().gs_gen_stencil27(grid, seed, C.byref(row), C.byref(col), C.byref(val),
                                     C.byref(n), C.byref(nnz)), "gs_gen_stencil27")
    return _finish(row, col, val, n.value, nnz.value)


def banded(nrows: int, half_bw: int, min_len: int, max_len: int, seed: int):
    """Banded random matrix: U[min_len, max_len] entries per row inside the band."""
    row, col, val = L.UINp(), L.UINp(), L.FPTp()
    got = L.UIN()
    L.check(L.lib().gs_gen_banded(nrows, half_bw, min_len, max_len, seed, C.byref(row),
                                  C.byref(col), C.byref(val), C.byref(got)), "gs_gen_banded")
    return _finish(row, col, val, nrows, got.value)


def vector(n: int, dist: str = "uniform", lo: float = -1.0, hi: float = 1.0, seed: int = 0):
    """uniform [lo, hi) or standard normal entries, one counter-based stream per entry."""
    v = np.empty(n, np.float64)
    L.check(L.lib().gs_gen_vector(n, 0 if dist == "uniform" else 1, lo, hi, seed,
                                  v.ctypes.data_as(L.FPTp)), "gs_gen_vector")
    return v


def banded_batch(count: int = 256, seed: int = 3):
    """The batched workload: `count` banded matrices with rows log-uniform in
    [1000, 200000], half-bandwidth U[16, 256], U[5, 60] entries per row inside the band,
    values N(0,1) (matrix i from seed 1000 * seed + i), each with U[1, 32] right-hand sides.
    Returns a list of (row, col, val, k)."""
    rng = np.random.default_rng(seed)
    nrows = np.exp(rng.uniform(np.log(1000), np.log(200000), count)).astype(np.int64)
    hbw = rng.integers(16, 257, count)
    ks = rng.integers(1, 33, count)
    out = []
    for i in range(count):
        row, col, val = banded(int(nrows[i]), int(hbw[i]), 5, 60, seed=1000 * seed + i)
        out.append((row, col, val, int(ks[i])))
    return out


def batch_rhs(i: int, ncols: int, k: int, seed: int = 3, dtype=np.float32):
    """Right-hand sides of matrix i of banded_batch: [ncols, k] N(0,1) entries."""
    g = np.random.default_rng([seed, i])
    return g.standard_normal((ncols, k)).astype(dtype)
