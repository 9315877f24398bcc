"""ORACLE TEST INFRASTRUCTURE -- the benchmark's seeded workloads for the reference arm.

``bench.py --impl reference`` times the reference's own CPU SpMV and must not load the
engine library for anything, not even to build its inputs.  This module binds
``oracle/_build/libgs_workload.so``: the engine's generator source
(``gpu_spmv_b200/csrc/gs_gen.cpp``) compiled on its own by ``make -C oracle port`` with the
engine's host flags.  The same seed gives the same bytes as ``gpu_spmv_b200.matgen``
(``tests/test_matgen.py`` checks it), so both arms of the benchmark multiply the same matrix
by the same vector.

Arrays are numpy: row/col uint32, val float64 (the reference's UIN / FPT).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
WORKLOAD_SO = os.path.join(HERE, "_build", "libgs_workload.so")

_UIN = C.c_uint32
_UINp = C.POINTER(_UIN)
_FPTp = C.POINTER(C.c_double)
_lib = None
_lock = threading.Lock()


def lib() -> C.CDLL:
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(WORKLOAD_SO):
                subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
            L = C.CDLL(WORKLOAD_SO)
            P = C.POINTER
            sig = {
                "gs_gen_laplacian2d": [_UIN, P(_UINp), P(_UINp), P(_FPTp), P(_UIN), P(_UIN)],
                "gs_gen_powerlaw": [_UIN, C.c_uint64, C.c_double, C.c_double, _UIN, C.c_uint64,
                                    P(_UINp), P(_UINp), P(_FPTp), P(_UIN)],
                "gs_gen_stencil27": [_UIN, C.c_uint64, P(_UINp), P(_UINp), P(_FPTp), P(_UIN),
                                     P(_UIN)],
                "gs_gen_banded": [_UIN, _UIN, _UIN, _UIN, C.c_uint64, P(_UINp), P(_UINp),
                                  P(_FPTp), P(_UIN)],
                "gs_gen_vector": [C.c_uint64, C.c_int, C.c_double, C.c_double, C.c_uint64,
                                  _FPTp],
            }
            for name, args in sig.items():
                f = getattr(L, name)
                f.restype = C.c_int
                f.argtypes = args
            L.gs_free_host.restype = None
            L.gs_free_host.argtypes = [C.c_void_p]
            _lib = L
    return _lib


def _check(st, where):
    if st != 0:
        raise RuntimeError(f"{where} failed with status {st}")


def _take(ptr, n, dtype):
    out = np.zeros(0, dtype) if n == 0 else np.ctypeslib.as_array(ptr, shape=(n,)).copy().view(dtype)
    lib().gs_free_host(C.cast(ptr, C.c_void_p))
    return out


def _finish(row, col, val, n, nnz):
    return (_take(row, n + 1, np.uint32), _take(col, nnz, np.uint32),
            _take(val, nnz, np.float64))


def laplacian2d(grid: int = 512):
    row, col, val, n, nnz = _UINp(), _UINp(), _FPTp(), _UIN(), _UIN()
    _check(lib().gs_gen_laplacian2d(grid, C.byref(row), C.byref(col), C.byref(val), C.byref(n),
                                    C.byref(nnz)), "gs_gen_laplacian2d")
    return _finish(row, col, val, n.value, nnz.value)


def powerlaw(nrows: int = 4194304, nnz: int = 67108864, mu: float = 2.5, sigma: float = 1.2,
             max_len: int = 10000, seed: int = 1):
    row, col, val, got = _UINp(), _UINp(), _FPTp(), _UIN()
    _check(lib().gs_gen_powerlaw(nrows, nnz, mu, sigma, max_len, seed, C.byref(row),
                                 C.byref(col), C.byref(val), C.byref(got)), "gs_gen_powerlaw")
    return _finish(row, col, val, nrows, got.value)


def stencil27(grid: int = 160, seed: int = 2):
    row, col, val, n, nnz = _UINp(), _UINp(), _FPTp(), _UIN(), _UIN()
    _check(lib().gs_gen_stencil27(grid, seed, C.byref(row), C.byref(col), C.byref(val),
                                  C.byref(n), C.byref(nnz)), "gs_gen_stencil27")
    return _finish(row, col, val, n.value, nnz.value)


def banded(nrows: int, half_bw: int, min_len: int, max_len: int, seed: int):
    row, col, val, got = _UINp(), _UINp(), _FPTp(), _UIN()
    _check(lib().gs_gen_banded(nrows, half_bw, min_len, max_len, seed, C.byref(row),
                               C.byref(col), C.byref(val), C.byref(got)), "gs_gen_banded")
    return _finish(row, col, val, nrows, got.value)


def vector(n: int, dist: str = "uniform", lo: float = -1.0, hi: float = 1.0, seed: int = 0):
    v = np.empty(n, np.float64)
    _check(lib().gs_gen_vector(n, 0 if dist == "uniform" else 1, lo, hi, seed,
                               v.ctypes.data_as(_FPTp)), "gs_gen_vector")
    return v
