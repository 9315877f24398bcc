"""The reference's second API generation (gpuSpmv_header.h) through gs2_*.

CPU: the two reference generations, both compiled unchanged, produce the same AXC, K1 and
AXT NOC/UNC arrays (which is what lets gs2_* reuse the first generation's converters), and
gs2_printMatrixStats writes the second generation's .sta file byte for byte.
GPU: every gs2_* converter output equals the compiled second generation's, bit for bit,
and the entry points score within round-off against its CPU product."""
import ctypes as C
import os

import numpy as np
import pytest

from mats import CASES, case

ref_needed = pytest.mark.skipif(
    not (os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle", "_ref",
                                     "libref_gen2.so"))),
    reason="oracle/_ref/libref_gen2.so not built (needs the reference sources)")

NOC = [(1, 32), (1, 16), (1, 4), (4, 32), (8, 32)]


class Csr2:
    """A gs2_matCSR over numpy arrays (kept alive here)."""

    def __init__(self, row, col, val):
        from gpu_spmv_b200 import _lib as L

        self.row = np.ascontiguousarray(row, np.uint32)
        self.col = np.ascontiguousarray(col, np.uint32)
        self.val = np.ascontiguousarray(val, np.float64)
        self.rl = np.diff(self.row).astype(np.uint32)
        m = L.Gen2MatCSR()
        m.nrows, m.nnz = len(self.row) - 1, len(self.col)
        m.val = self.val.ctypes.data_as(L.FPTp)
        m.row = self.row.ctypes.data_as(L.UINp)
        m.col = self.col.ctypes.data_as(L.UINp)
        m.rl = (self.rl if len(self.rl) else np.zeros(1, np.uint32)).ctypes.data_as(L.UINp)
        self.m = m


def _arr(ptr, n, dt):
    return np.ctypeslib.as_array(ptr, (n,)).astype(dt).copy() if n else np.zeros(0, dt)


@ref_needed
@pytest.mark.parametrize("name", CASES)
def test_reference_generations_share_layouts(name):
    from oracle.oracle import Ref, Ref2

    R, R2 = Ref(), Ref2()
    rng = np.random.default_rng(1)
    row, col, val = case(name, rng)
    n = len(row) - 1
    x = np.arange(max(n, int(col.max()) + 1), dtype=np.float64)
    a1, a2 = R.axc(row, col, val, x, hbs=32), R2.axc(row, col, val, x)
    assert np.array_equal(a1["ax"], a2["ax"]) and np.array_equal(a1["brp"], a2["brp"])
    k1, k2 = R.k1(row, col, val, x), R2.k1(row, col, val, x)
    for key in ("permi", "nmc", "chp", "val", "col"):
        assert np.array_equal(k1[key][:len(k2[key])], k2[key]), key
    for th, thw in NOC:
        t1 = R.axt(row, col, val, x, thw, th, "UNC")
        t2 = R2.axt(row, col, val, x, thw, th, "NOC")
        assert (t1["tileN"], t1["lenAX"], t1["lenSEC"]) == (t2["tileN"], t2["lenAX"], t2["lenSEC"])
        assert np.array_equal(t1["ax"], t2["ax"]) and np.array_equal(t1["sec"], t2["sec"])
        assert np.array_equal(t1["con"][:n], t2["con"])


@ref_needed
def test_gen2_stats_file(tmp_path):
    from gpu_spmv_b200 import _lib as L
    from oracle.oracle import Ref2

    rng = np.random.default_rng(3)
    row, col, val = case("powerlaw_small", rng)
    path = str(tmp_path / "m.bin")
    sta = str(tmp_path / "m.sta")
    _, st = Ref2().stats(path, row, col, val)
    want = open(sta, "rb").read()
    os.remove(sta)
    h = Csr2(row, col, val)
    L.lib().gs2_printMatrixStats(path.encode(), C.byref(h.m))
    assert open(sta, "rb").read() == want
    assert (h.m.rmin, h.m.rmax, h.m.bw) == (st["rmin"], st["rmax"], st["bw"])
    assert h.m.rave == st["rave"] and h.m.rsd == st["rsd"]
    assert np.array_equal(h.rl, np.diff(row))


# the reference API is square-only (x has nrows entries): single_row (1 x 50) is left out
SQUARE = [c for c in CASES if c != "single_row"]


@ref_needed
@pytest.mark.gpu
@pytest.mark.parametrize("name", SQUARE)
def test_gen2_converters_and_entry_points(name):
    from gpu_spmv_b200 import _lib as L
    from oracle.oracle import Ref2

    lib, R2 = L.lib(), Ref2()
    lib.gs_set_num_ite(3)
    rng = np.random.default_rng(7)
    row, col, val = case(name, rng)
    n = len(row) - 1
    x = np.arange(max(n, int(col.max()) + 1), dtype=np.float64)  # initVec, as gpuSpmv_main
    h = Csr2(row, col, val)
    ref = R2.cf_csr(row, col, val, x)
    xp = x.ctypes.data_as(L.FPTp)
    rp = ref.ctypes.data_as(L.FPTp)

    def good(res, want):
        assert res.name.decode() == want
        assert res.sErr.rErr <= 1e-12, (want, res.sErr.rErr)

    good(lib.gs2_test_gk_CSR(256, h.m, xp, rp), "gk_CSR")
    good(lib.gs2_test_cf_CSR(h.m, xp, rp), "cf_CSR")
    # AXC
    a = L.Gen2MatAXC()
    fd = lib.gs2_getFormatDataAXC(1, h.m, xp, C.byref(a))
    r = R2.axc(row, col, val, x)
    assert (a.lenAX, a.lenBRP) == (r["lenAX"], r["lenBRP"])
    assert np.array_equal(_arr(a.ax, a.lenAX, np.float64), r["ax"])
    assert np.array_equal(_arr(a.brp, a.lenBRP, np.uint32), r["brp"])
    assert (fd.name.decode(), fd.mfp, fd.beta) == (r["fd"]["name"], r["fd"]["mfp"], r["fd"]["beta"])
    good(lib.gs2_test_gk_AXC(256, a, rp), "gk_AXC")
    # K1
    k = L.StrMatK1()
    fd = lib.gs2_getFormatDataK1(256, h.m, xp, C.byref(k))
    r = R2.k1(row, col, val, x)
    assert (k.chunkNum, k.lenVC) == (r["chunkNum"], r["lenVC"])
    for key, ptr, cnt, dt in (("permi", k.permi, k.chunkNum * 32, np.uint32),
                              ("nmc", k.nmc, k.chunkNum, np.uint32),
                              ("chp", k.chp, k.chunkNum, np.uint32),
                              ("val", k.val, k.lenVC, np.float64),
                              ("col", k.col, k.lenVC, np.uint32)):
        assert np.array_equal(_arr(ptr, cnt, dt), r[key]), key
    assert (fd.name.decode(), fd.mfp, fd.beta) == (r["fd"]["name"], r["fd"]["mfp"], r["fd"]["beta"])
    good(lib.gs2_test_gk_K1(256, k, xp, rp), "gk_K1")
    # AXT
    for mode, th, thw, bs in [("NOC", t, w, 256) for t, w in NOC] + \
            [("COM", 1, 32, 256), ("COM", 1, 32, 1024), ("COM", 4, 32, 256)]:
        t = L.Gen2MatAXT()
        fd = lib.gs2_getFormatDataAXT(1, bs, thw, th, mode.encode(), h.m, xp, C.byref(t))
        r = R2.axt(row, col, val, x, thw, th, mode, bs=bs)
        key = (mode, th, thw, bs)
        assert (t.tileN, t.lenAX, t.lenSEC, t.lenCON, t.logTH, t.log) == \
            (r["tileN"], r["lenAX"], r["lenSEC"], r["lenCON"], r["logTH"], r["log"]), key
        assert np.array_equal(_arr(t.ax, t.lenAX, np.float64), r["ax"]), key
        assert np.array_equal(_arr(t.sec, t.lenSEC, np.uint32), r["sec"]), key
        assert np.array_equal(_arr(t.con, t.lenCON, np.uint32), r["con"]), key
        assert (fd.name.decode(), fd.mfp, fd.beta) == \
            (r["fd"]["name"], r["fd"]["mfp"], r["fd"]["beta"]), key
        if mode == "NOC" and th == 1:
            good(lib.gs2_test_gk_AXT_NOC_H1(256, t, rp), f"gk_AXT_NOC_H1_HW{thw}")
        elif mode == "NOC":
            good(lib.gs2_test_gk_AXT_NOC(256, t, rp), f"gk_AXT_NOC_H{th}_HW{thw}")
        elif th == 1:
            good(lib.gs2_test_gk_AXT_COM_H1(256, t, rp), f"gk_AXT_COM_H1_HW{thw}")
    lib.gs_set_num_ite(250)
