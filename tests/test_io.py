"""Matrix I/O and statistics of the drop-in layer (host code, no GPU): the .bin/.csr readers
(cudaSpmv.cu:265-328), the .bin writer, and printMatrixStats (cudaSpmv.cu:332-381)
against the reference's own statistics."""
import ctypes as C
import os

import numpy as np

from gpu_spmv_b200 import _lib as L
from gpu_spmv_b200 import refapi as R
from mats import case


def test_bin_roundtrip_and_stats(tmp_path, port):
    rng = np.random.default_rng(9)
    row, col, val = case("mixed", rng)
    h = R.csr_struct(row, col, val)
    path = str(tmp_path / "m.bin")
    assert L.lib().matrixWritingBin(path.encode(), C.byref(h.s)) == 0
    m = L.lib().matrixReading(path.encode())
    n = m.nrows
    assert n == len(row) - 1 and m.nnz == len(col)
    assert np.array_equal(np.ctypeslib.as_array(m.row, (n + 1,)), row)
    assert np.array_equal(np.ctypeslib.as_array(m.col, (m.nnz,)), col)
    assert np.array_equal(np.ctypeslib.as_array(m.val, (m.nnz,)), val)
    L.lib().printMatrixStats(path.encode(), C.byref(m))
    rl, st = port.row_stats(row, col)
    assert np.array_equal(np.ctypeslib.as_array(m.rl, (n,)), rl)
    assert (m.rmin, m.rmax, m.bw) == (st["rmin"], st["rmax"], st["bw"])
    assert m.rave == st["rave"] and m.rsd == st["rsd"]
    sta = open(str(tmp_path / "m.sta")).read()
    assert "matrix's statistics" in sta and f"{n}" in sta
    fd = L.lib().getFormatDataCSR(C.byref(m))
    assert fd.name == b"fcsr" and fd.beta == 1.0
    assert fd.mfp == m.nnz * 8 + m.nnz * 4 + (n + 1) * 4 + n * 8
    assert np.array_equal(np.ctypeslib.as_array(m.rowStart, (n,)), row[:-1])
    assert np.array_equal(np.ctypeslib.as_array(m.rowEnd, (n,)), row[1:])


def test_stats_match_reference(tmp_path, ref):
    rng = np.random.default_rng(10)
    row, col, val = case("powerlaw_small", rng)
    h = R.csr_struct(row, col, val)
    path = str(tmp_path / "p.bin")
    L.lib().matrixWritingBin(path.encode(), C.byref(h.s))
    m = L.lib().matrixReading(path.encode())
    L.lib().printMatrixStats(path.encode(), C.byref(m))
    rl, st = ref.stats(str(tmp_path / "q.bin"), row, col, val)
    assert (m.rmin, m.rmax, m.bw) == (st["rmin"], st["rmax"], st["bw"])
    assert m.rave == st["rave"] and m.rsd == st["rsd"]


def test_csr_text_reader(tmp_path):
    p = tmp_path / "t.csr"
    p.write_text("3 4\n1.5 0\n-2.0 2\n3.25 1\n4.0 2\n0 2 3 4\n")
    m = L.lib().matrixReading(str(p).encode())
    assert (m.nrows, m.nnz) == (3, 4)
    assert np.array_equal(np.ctypeslib.as_array(m.val, (4,)), [1.5, -2.0, 3.25, 4.0])
    assert np.array_equal(np.ctypeslib.as_array(m.row, (4,)), [0, 2, 3, 4])


def test_reader_rejects_unknown_extension(tmp_path):
    p = tmp_path / "x.mtx"
    p.write_text("")
    m = L.lib().matrixReading(str(p).encode())
    assert m.nrows == 0 and not m.val
    assert b"extension" in L.lib().gs_last_error()
