"""The CPU oracle is pinned before anything is checked against it:
  * the C restatement (oracle/spmv_oracle.c) reproduces the golden fixtures that the
    reference's own compiled code produced (tests/golden/*.npz), bit for bit;
  * where oracle/_ref is built, the restatement equals the live reference on every test
    matrix and every converter parameter set.
"""
import glob
import os

import numpy as np
import pytest

from mats import AXT_PARAMS, CASES, case

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _slots_of(ax_len, w):
    s = np.arange(ax_len // 2)
    return (s // w) * 2 * w + s % w


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_port_matches_golden(port, path):
    g = np.load(path)
    row, col, val, x = g["row"], g["col"], g["val"], g["x"]
    n = len(row) - 1
    xi = np.arange(n, dtype=np.float64)
    # CPU CSR SpMV: exact (same operation order, no FMA)
    assert np.array_equal(port.csr_spmv(row, col, val, x), g["y_ncsr"])
    assert np.array_equal(port.csr_spmv(row, col, val, x), g["y_cpuSpmvCSR"])
    assert np.array_equal(port.csr_spmv(row, col, val, xi), g["y_ncsr_xi"])
    rl, st = port.row_stats(row, col)
    assert np.array_equal(rl, g["rl"])
    assert np.allclose([st["rmin"], st["rave"], st["rmax"], st["rsd"], st["bw"]], g["stats"],
                       rtol=0, atol=0)
    k = port.k1(row, col, val)
    for f in ("permi", "nmc", "chp", "val", "col"):
        assert np.array_equal(k[f], g[f"k1_{f}"]), f
    a = port.axc(row, col, val, x=xi, hbs=32)
    for f in ("brp", "ax", "mapx"):
        assert np.array_equal(a[f], g[f"axc_{f}"]), f
    for (mode, th, thw, bs) in AXT_PARAMS:
        key = f"axt_{mode}_{th}_{thw}_{bs}"
        t = port.axt(row, col, val, thw, th, mode, bs=bs, x=xi)
        d = t["dims"]
        assert [d.tileN, d.lenAX, d.lenSEC, d.lenCON, d.log, d.logTH] == list(g[key + "_dims"])
        assert np.array_equal(t["ax"], g[key + "_ax"]), key
        assert np.array_equal(t["sec"], g[key + "_sec"]), key
        assert np.array_equal(t["con"], g[key + "_con"]), key
        # native streams are the two halves of ax (x half == column index when x[i] = i)
        idx = _slots_of(len(t["ax"]), thw)
        assert np.array_equal(t["val"], g[key + "_ax"][idx])
        assert np.array_equal(t["col"].astype(np.float64), g[key + "_ax"][idx + thw])


@pytest.mark.parametrize("name", CASES)
def test_port_matches_live_reference(port, ref, name, rng):
    row, col, val = case(name, np.random.default_rng(sum(map(ord, name))))
    n = len(row) - 1
    ncols = max(n, int(col.max()) + 1 if len(col) else n)
    if ncols != n:
        pytest.skip("reference converters assume square matrices")
    xi = ref.init_vec(n)
    x = rng.uniform(-1, 1, n)
    assert np.array_equal(port.csr_spmv(row, col, val, x), ref.ncsr(row, col, val, x))
    k, kr = port.k1(row, col, val), ref.k1(row, col, val, xi)
    for f in ("permi", "nmc", "chp", "val", "col"):
        assert np.array_equal(k[f], kr[f]), f
    a, ar = port.axc(row, col, val, x=xi), ref.axc(row, col, val, xi)
    for f in ("brp", "ax", "mapx"):
        assert np.array_equal(a[f], ar[f]), f
    for (mode, th, thw, bs) in AXT_PARAMS:
        t = port.axt(row, col, val, thw, th, mode, bs=bs, x=xi)
        tr = ref.axt(row, col, val, xi, thw, th, mode, bs=bs)
        for f in ("ax", "sec", "con"):
            assert np.array_equal(t[f], tr[f]), (mode, th, thw, bs, f)


@pytest.mark.parametrize("name", CASES)
def test_port_layout_spmv_consistent(port, name, rng):
    """Every restated layout computes A x (within FP64 reordering error)."""
    row, col, val = case(name, np.random.default_rng(1 + sum(map(ord, name))))
    n = len(row) - 1
    ncols = max(n, int(col.max()) + 1 if len(col) else n)
    x = rng.uniform(-1, 1, ncols)
    y_true, mag = port.csr_truth(row, col, val, x)
    k = port.k1(row, col, val)
    assert np.all(np.abs(port.k1_spmv(k, x) - y_true) <= 1e-13 * mag + 0.0)
    for (mode, th, thw, bs) in AXT_PARAMS:
        if mode == "COM" and (th & (th - 1)):
            continue
        t = port.axt(row, col, val, thw, th, mode, bs=bs, x=x)
        assert np.all(np.abs(port.axt_spmv(t, x) - y_true) <= 1e-13 * mag), (mode, th, thw)
        assert np.all(np.abs(port.axt_spmv_baked(t) - y_true) <= 1e-13 * mag), (mode, th, thw)


def test_k1_permutation_is_stable_descending(port, rng):
    lens = rng.integers(0, 6, 4000)  # many ties
    from mats import csr_from_lengths

    row, col, val = csr_from_lengths(lens, 4000, rng)
    k = port.k1(row, col, val)
    p = k["permi"][:4000]
    rl = np.diff(row)[p]
    assert np.all(rl[:-1] >= rl[1:])
    ties = rl[:-1] == rl[1:]
    assert np.all(p[:-1][ties] < p[1:][ties])


def test_com_row0_header_is_zero(port):
    """The layout fact behind the reference defect in gaxtch1 (cudaSpmv.cu:2089): when row
    0 has one element, its COM header word is 0 and indistinguishable from 'no header'
    unless the decoder knows every segment block starts with a header."""
    row = np.array([0, 1, 3, 6], np.uint32)
    col = np.array([0, 0, 2, 0, 1, 2], np.uint32)
    val = np.arange(1, 7, dtype=np.float64)
    t = port.axt(row, col, val, 32, 1, "COM", bs=4)
    assert t["sec"][0] == 0
    x = np.array([1.0, 2.0, 3.0])
    assert np.array_equal(port.axt_spmv(t, x), port.csr_spmv(row, col, val, x))


@pytest.fixture(scope="module")
def powerlaw_64m():
    from gpu_spmv_b200 import matgen

    row, col, val = matgen.powerlaw(seed=1)
    x = matgen.vector(len(row) - 1, "uniform", -1.0, 1.0, seed=1001)
    return row, col, val, x


def test_restatement_equals_reference_at_benchmark_size(port, ref, powerlaw_64m):
    """The restated converters against the reference's own (compiled unchanged) on the
    headline power-law matrix, 4,194,304 rows and 67,108,864 nnz: K1 (cudaSpmv.cu:716-846,
    a stable sort of 4M rows with heavy length ties), AXT UNC tileH 4 and COM tileH 1
    (cudaSpmv.cu:1158-1566), bit for bit."""
    row, col, val, x = powerlaw_64m
    k_ref = ref.k1(row, col, val, x)
    k = port.k1(row, col, val)
    for f in ("permi", "nmc", "chp", "val", "col"):
        assert np.array_equal(k[f], k_ref[f]), f
    del k_ref, k
    for thw, th, mode in ((32, 4, "UNC"), (32, 1, "COM")):
        a_ref = ref.axt(row, col, val, x, thw, th, mode, threads=os.cpu_count() or 1)
        a = port.axt(row, col, val, thw, th, mode, x=x)
        for f in ("ax", "sec", "con"):
            assert np.array_equal(a[f], a_ref[f]), (mode, th, f)


@pytest.mark.parametrize("name", CASES)
def test_gen0_brick_formats_are_axc_and_axt_layouts(port, ref, name):
    """The first generation's brick formats (spmv_header.h, compiled unchanged) are layouts
    the restated converters already build, with bricks of HBRICK_SIZE = 16:
    AXCv0 = AXC hbs 16 (brp, ax; spmv_header.h:665-760); AXCv1 = AXT UNC tileH 1 tileHW 16
    (brp = con, rwp = sec; :851-960); AXBv0 = AXT COM tileH 1 tileHW 16 with a header word
    every 32 positions (hdr0 = sec, bs = 32; :1649-1727); AXBv1 = the same with a header
    every cudaBlockSize positions, hdr1 padded to a multiple of 32 words (:2299-2390)."""
    if ref.lib_spmv is None or not hasattr(ref.lib_spmv, "ref0_convert"):
        pytest.skip("first-generation oracle library not built")
    rng = np.random.default_rng(sum(map(ord, name)) + 5)
    row, col, val = case(name, rng)
    n = len(row) - 1
    x = rng.uniform(-1, 1, max(n, int(col.max()) + 1))
    a0 = ref.gen0("AXCv0", row, col, val, x)
    pa = port.axc(row, col, val, x=x, hbs=16)
    assert np.array_equal(a0["ax"], pa["ax"]) and np.array_equal(a0["brp"], pa["brp"])
    a1 = ref.gen0("AXCv1", row, col, val, x)
    pu = port.axt(row, col, val, 16, 1, "UNC", x=x)
    assert np.array_equal(a1["ax"], pu["ax"]) and np.array_equal(a1["brp"], pu["con"])
    assert np.array_equal(a1["rwp"], pu["sec"])
    b0 = ref.gen0("AXBv0", row, col, val, x)
    pc = port.axt(row, col, val, 16, 1, "COM", bs=32, x=x)
    assert np.array_equal(b0["ax"], pc["ax"]) and np.array_equal(b0["hdr"], pc["sec"])
    for cbs in (64, 256, 1024):
        b1 = ref.gen0("AXBv1", row, col, val, x, cbs=cbs)
        pc = port.axt(row, col, val, 16, 1, "COM", bs=cbs, x=x)
        assert b1["blockLog"] == cbs.bit_length() - 1
        assert np.array_equal(b1["ax"], pc["ax"])
        assert len(b1["hdr"]) == (len(pc["sec"]) + 31) // 32 * 32
        assert np.array_equal(b1["hdr"][:len(pc["sec"])], pc["sec"])
        assert not b1["hdr"][len(pc["sec"]):].any()
    assert (a0["name"], a1["name"], b0["name"]) == ("AXCv0", "AXCv1", "AXBv0")
