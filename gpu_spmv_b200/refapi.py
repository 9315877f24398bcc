"""Python access to the drop-in layer: the reference program's structs and entry points
(cudaSpmv.cu names) as exported by the engine library.

``csr_struct`` builds a ``str_matCSR`` over numpy arrays (kept alive by the returned
holder); the converters and ``test_*`` entry points are then called exactly as the
reference's main() calls them (cudaSpmv.cu:2319-2417).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class CSRHolder:
    """A str_matCSR plus the numpy arrays it points into."""

    def __init__(self, row, col, val, name="matrix"):
        self.row = np.ascontiguousarray(row, dtype=np.uint32)
        self.col = np.ascontiguousarray(col, dtype=np.uint32)
        self.val = np.ascontiguousarray(val, dtype=np.float64)
        n = len(self.row) - 1
        self.rl = np.diff(self.row).astype(np.uint32)
        s = L.StrMatCSR()
        s.name = name.encode()[:47]
        s.nrows = n
        s.nnz = len(self.col)
        s.val = self.val.ctypes.data_as(L.FPTp)
        s.col = self.col.ctypes.data_as(L.UINp)
        s.row = self.row.ctypes.data_as(L.UINp)
        s.rl = self.rl.ctypes.data_as(L.UINp)
        self.s = s


def csr_struct(row, col, val, name="matrix") -> CSRHolder:
    return CSRHolder(row, col, val, name)


def f64p(a: np.ndarray):
    return a.ctypes.data_as(L.FPTp)


def arr_u32(ptr, n) -> np.ndarray:
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, np.uint32)


def arr_f64(ptr, n) -> np.ndarray:
    return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, np.float64)


def free_struct_arrays(st, fields):
    libc = C.CDLL(None)
    libc.free.argtypes = [C.c_void_p]
    for f in fields:
        p = getattr(st, f)
        if p:
            libc.free(C.cast(p, C.c_void_p))
        setattr(st, f, None)


def k1_arrays(k: L.StrMatK1) -> dict:
    return dict(permi=arr_u32(k.permi, (k.chunkNum + 1) * 32), nmc=arr_u32(k.nmc, k.chunkNum),
                chp=arr_u32(k.chp, k.chunkNum), val=arr_f64(k.val, k.lenVC),
                col=arr_u32(k.col, k.lenVC))


def axc_arrays(a: L.StrMatAXC) -> dict:
    return dict(ax=arr_f64(a.ax, a.lenAX), brp=arr_u32(a.brp, a.lenBRP),
                mapx=arr_u32(a.mapx, a.lenMAPX))


def axt_arrays(a: L.StrMatAXT) -> dict:
    return dict(ax=arr_f64(a.ax, a.lenAX), sec=arr_u32(a.sec, a.lenSEC),
                con=arr_u32(a.con, a.lenCON + 1))


def last_y(n: int) -> np.ndarray:
    """y of this thread's most recent drop-in test_* product (row order)."""
    out = np.zeros(n, np.float64)
    got = L.lib().gs_dropin_last_y(f64p(out), n)
    if got != n:
        raise RuntimeError(f"the last drop-in product had {got} rows, expected {n}")
    return out
