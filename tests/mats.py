"""Small CSR test matrices (numpy) covering the edge cases the reference's layouts have:
empty rows (including row 0 and the last row), a row 0 of length 1 (the COM header word
that equals 0), rows exactly tileHW / multiples of tileH long, rows longer than a warp's
share, an all-empty K1 chunk, a single row, and a dense row."""
from __future__ import annotations

import numpy as np


def csr_from_lengths(lens, ncols, rng, values="normal"):
    lens = np.asarray(lens, dtype=np.int64)
    n = len(lens)
    row = np.zeros(n + 1, np.uint32)
    row[1:] = np.cumsum(lens)
    cols = []
    for l in lens:
        cols.append(np.sort(rng.choice(ncols, size=int(l), replace=False)))
    col = (np.concatenate(cols) if cols else np.zeros(0)).astype(np.uint32)
    nnz = int(row[-1])
    if values == "normal":
        val = rng.standard_normal(nnz)
    else:
        val = rng.uniform(-1, 1, nnz)
    return row, col, val


def case(name, rng):
    """Named square test matrices."""
    if name == "mixed":
        n = 700
        lens = rng.integers(0, 45, n)
        lens[0] = 1
        lens[3] = 0
        lens[10] = 32
        lens[11] = 64
        lens[12] = 16
        lens[13] = 600
        lens[-1] = 0
        return csr_from_lengths(lens, n, rng)
    if name == "row0_empty":
        n = 300
        lens = rng.integers(0, 12, n)
        lens[:5] = 0
        return csr_from_lengths(lens, n, rng)
    if name == "k1_empty_chunk":
        n = 200
        lens = rng.integers(1, 9, n)
        lens[64:] = 0  # sorted descending: chunks 2.. are all empty
        return csr_from_lengths(lens, n, rng)
    if name == "single_row":
        return csr_from_lengths([37], 50, rng)
    if name == "dense_row":
        n = 3000
        lens = rng.integers(1, 6, n)
        lens[7] = 2900
        return csr_from_lengths(lens, n, rng)
    if name == "powerlaw_small":
        n = 5000
        L = np.clip(rng.lognormal(2.5, 1.2, n), 1, 2000)
        lens = np.clip(np.rint(L * 0.64), 1, 2000).astype(np.int64)
        return csr_from_lengths(lens, n, rng)
    if name == "laplacian":
        g = 24
        n = g * g
        rows, cols, vals = [0], [], []
        for r in range(n):
            i, j = divmod(r, g)
            ent = []
            if i > 0: ent.append((r - g, -1.0))
            if j > 0: ent.append((r - 1, -1.0))
            ent.append((r, 4.0))
            if j + 1 < g: ent.append((r + 1, -1.0))
            if i + 1 < g: ent.append((r + g, -1.0))
            for c, v in ent:
                cols.append(c)
                vals.append(v)
            rows.append(len(cols))
        return (np.array(rows, np.uint32), np.array(cols, np.uint32), np.array(vals))
    raise KeyError(name)


CASES = ["mixed", "row0_empty", "k1_empty_chunk", "single_row", "dense_row", "powerlaw_small",
         "laplacian"]

# (mode, tileH, tileHW, bs) parameter sets of the reference's main (cudaSpmv.cu:2349-2360)
# plus the tileH in {2, 8} of the benchmark configuration
AXT_PARAMS = [("UNC", 1, 16, 256), ("UNC", 1, 8, 256), ("UNC", 1, 4, 256), ("UNC", 1, 32, 256),
              ("UNC", 2, 32, 256), ("UNC", 4, 32, 256), ("UNC", 6, 32, 256),
              ("UNC", 8, 32, 256), ("UNC", 10, 32, 256), ("UNC", 12, 32, 256),
              ("UNC", 4, 16, 256), ("COM", 1, 32, 256), ("COM", 1, 32, 64),
              ("COM", 4, 32, 256), ("COM", 8, 32, 256), ("COM", 16, 32, 256)]


def within_bound(y, y_ref, abs_ax, rel=1e-13):
    """max |y - y_ref| <= rel * (|A||x|)_i, row by row."""
    return np.all(np.abs(y - y_ref) <= rel * abs_ax)
