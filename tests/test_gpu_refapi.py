"""Drop-in layer on the GPU, called the way the reference's main() calls it
(cudaSpmv.cu:2319-2417): the converters return host arrays identical to the reference's
own (golden fixtures made by the compiled reference), and every test_* entry point
returns y within 1e-13 * (|A||x|)_i of the reference's CPU path."""
import ctypes as C
import glob
import os

import numpy as np
import pytest

from mats import AXT_PARAMS, case

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


@pytest.fixture(scope="module")
def lib():
    from gpu_spmv_b200 import _lib as L

    lib = L.lib()
    lib.gs_set_num_ite(3)
    yield lib
    lib.gs_set_num_ite(250)


def _bound(port, row, col, val, x):
    _, mag = port.csr_truth(row, col, val, x)
    return 1e-13 * mag.max()


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
def test_dropin_converters_match_reference(lib, port, path):
    from gpu_spmv_b200 import _lib as L
    from gpu_spmv_b200 import refapi as R

    g = np.load(path)
    row, col, val = g["row"], g["col"], g["val"]
    n = len(row) - 1
    h = R.csr_struct(row, col, val, name="golden.bin")
    xi = np.zeros(n)
    lib.init_vec(1, n, R.f64p(xi))
    assert np.array_equal(xi, np.arange(n, dtype=np.float64))
    y_ref = g["y_ncsr_xi"]
    tol = _bound(port, row, col, val, xi)

    k = L.StrMatK1()
    fd = lib.getFormatDataK1(32, h.s, R.f64p(xi), C.byref(k))
    assert fd.name == b"fk1"
    ka = R.k1_arrays(k)
    for f in ("permi", "nmc", "chp", "val", "col"):
        assert np.array_equal(ka[f], g[f"k1_{f}"]), f
    res = lib.test_gk1(256, k, R.f64p(xi), R.f64p(y_ref))
    assert res.name == b"gk1" and res.et > 0 and res.sErr.aErr <= tol

    a = L.StrMatAXC()
    fd = lib.getFormatDataAXC(1, 32, h.s, R.f64p(xi), C.byref(a))
    assert fd.name == b"faxc"
    aa = R.axc_arrays(a)
    for f in ("brp", "ax", "mapx"):
        assert np.array_equal(aa[f], g[f"axc_{f}"]), f
    res = lib.test_gaxc(256, a, R.f64p(y_ref))
    assert res.name == b"gaxc" and res.sErr.aErr <= tol

    for (mode, th, thw, bs) in AXT_PARAMS:
        key = f"axt_{mode}_{th}_{thw}_{bs}"
        t = L.StrMatAXT()
        fd = lib.getFormatDataAXT(1, bs, thw, th, mode.encode(), h.s, R.f64p(xi), C.byref(t))
        assert fd.name != b"error", lib.gs_last_error()
        ta = R.axt_arrays(t)
        for f in ("ax", "sec", "con"):
            assert np.array_equal(ta[f], g[key + "_" + f]), (key, f)
        dims = [t.tileN, t.lenAX, t.lenSEC, t.lenCON, t.log, t.logTH]
        assert dims == list(g[key + "_dims"]), key
        assert t.mode == mode.encode() and t.tileHW == thw and t.tileH == th and t.bs == bs
        if mode == "UNC" and th == 1:
            fn = {16: lib.test_gaxtuh1hw16w, 8: lib.test_gaxtuh1hw08w, 4: lib.test_gaxtuh1hw04w}
            res = fn.get(thw, lib.test_gaxtuh1hw16w)(128, 256, t, R.f64p(y_ref))
            assert res.name.startswith(b"gaxtuh1hw"), res.name
        elif mode == "UNC":
            res = lib.test_gaxtuh(2, 256, t, R.f64p(y_ref))
            assert res.name == f"gaxtuh{th}tpw2".encode()
        elif th == 1:
            res = lib.test_gaxtch1(bs, t, R.f64p(y_ref))
            assert res.name == f"gaxtch1bs{bs}".encode()
        else:
            res = lib.test_gaxtch(256, t, R.f64p(y_ref))
            assert res.name == f"gaxtch{th}".encode()
        assert res.sErr.aErr <= tol, (key, res.sErr.aErr, tol)
        R.free_struct_arrays(t, ("ax", "sec", "con"))


def test_dropin_csr_entry_points(lib, port):
    from gpu_spmv_b200 import _lib as L
    from gpu_spmv_b200 import refapi as R

    rng = np.random.default_rng(3)
    row, col, val = case("powerlaw_small", rng)
    n = len(row) - 1
    h = R.csr_struct(row, col, val)
    x = rng.uniform(-1, 1, n)
    y_ref = port.csr_spmv(row, col, val, x)
    tol = _bound(port, row, col, val, x)
    y = np.zeros(n)
    lib.ncsr(8, h.s, R.f64p(x), R.f64p(y))
    _, mag = port.csr_truth(row, col, val, x)
    assert np.all(np.abs(y - y_ref) <= 1e-13 * mag)
    res = lib.test_gcsr(256, h.s, R.f64p(x), R.f64p(y_ref))
    assert res.name == b"gcsr" and res.sErr.aErr <= tol and res.flops > 0
    res = lib.test_gcucsr(h.s, R.f64p(x), R.f64p(y_ref))
    assert res.name == b"gcucsr"
    assert res.sErr.aErr <= 1e-12 * np.abs(y_ref).max()
    e = L.StrErr()
    lib.get_errors(n, R.f64p(y_ref), R.f64p(y), C.byref(e))
    assert (e.aErr, e.rErr, e.pos)[0] == port.get_errors(y_ref, y)[0]


def test_dropin_errors_do_not_exit(lib):
    from gpu_spmv_b200 import _lib as L
    from gpu_spmv_b200 import refapi as R

    h = R.csr_struct(np.array([0, 1], np.uint32), np.array([0], np.uint32), np.ones(1))
    t = L.StrMatAXT()
    fd = lib.getFormatDataAXT(1, 256, 32, 1, b"BAD", h.s, R.f64p(np.zeros(1)), C.byref(t))
    assert fd.name == b"error" and b"mode" in lib.gs_last_error()
    # a UNC entry point handed a COM matrix reports an error result instead of exiting
    fd = lib.getFormatDataAXT(1, 256, 32, 1, b"COM", h.s, R.f64p(np.zeros(1)), C.byref(t))
    res = lib.test_gaxtuh1hw16w(64, 256, t, R.f64p(np.zeros(1)))
    assert res.name == b"error"


def _dropin_inputs(name):
    rng = np.random.default_rng(7)
    if name.endswith(".npz"):
        g = np.load(name)
        row, col, val = g["row"], g["col"], g["val"]
        x = np.arange(len(row) - 1, dtype=np.float64)  # init_vec: x[i] = i
    else:
        row, col, val = case(name, rng)
        x = rng.uniform(-1, 1, len(row) - 1)
    return row, col, val, x


@pytest.mark.parametrize("name", GOLDEN + ["powerlaw_small", "mixed", "dense_row"],
                         ids=[os.path.basename(p) for p in GOLDEN] +
                         ["powerlaw_small", "mixed", "dense_row"])
def test_dropin_products_per_row_and_metrics(lib, port, ref, name):
    """Every drop-in test_* entry point's y, read back row by row, within
    1e-13 (|A||x|)_i of the reference's CPU loop with its sign (get_errors compares
    magnitudes only, cudaSpmv.cu:474-495); and every converter's format metrics (name, mfp,
    beta) equal to the compiled reference's getFormatData* (cudaSpmv.cu:826-845, 1050-1061,
    1558-1565)."""
    from gpu_spmv_b200 import _lib as L
    from gpu_spmv_b200 import refapi as R

    row, col, val, x = _dropin_inputs(name)
    n = len(row) - 1
    h = R.csr_struct(row, col, val)
    y_ref = port.csr_spmv(row, col, val, x)
    _, mag = port.csr_truth(row, col, val, x)

    def check(res, what):
        assert res.name != b"error", (what, lib.gs_last_error())
        y = R.last_y(n)
        err = np.abs(y - y_ref)
        assert np.all(err <= 1e-13 * mag), (what, float(np.max(err / np.maximum(mag, 1e-300))))

    check(lib.test_gcsr(256, h.s, R.f64p(x), R.f64p(y_ref)), "gcsr")

    k = L.StrMatK1()
    fd = lib.getFormatDataK1(32, h.s, R.f64p(x), C.byref(k))
    rk = ref.k1(row, col, val, x)
    assert (fd.name, fd.mfp, fd.beta) == (b"fk1", rk["fd"][0], rk["fd"][1])
    check(lib.test_gk1(256, k, R.f64p(x), R.f64p(y_ref)), "gk1")
    R.free_struct_arrays(k, ("permi", "nmc", "chp", "val", "col"))

    a = L.StrMatAXC()
    fd = lib.getFormatDataAXC(1, 32, h.s, R.f64p(x), C.byref(a))
    ra = ref.axc(row, col, val, x, hbs=32)
    assert (fd.name, fd.mfp, fd.beta) == (b"faxc", ra["fd"][0], ra["fd"][1])
    check(lib.test_gaxc(256, a, R.f64p(y_ref)), "gaxc")
    R.free_struct_arrays(a, ("ax", "brp", "mapx"))

    for (mode, th, thw, bs) in AXT_PARAMS + [("COM", 2, 32, 256)]:
        t = L.StrMatAXT()
        fd = lib.getFormatDataAXT(1, bs, thw, th, mode.encode(), h.s, R.f64p(x), C.byref(t))
        rt = ref.axt(row, col, val, x, thw, th, mode, bs=bs)
        key = (mode, th, thw, bs)
        assert fd.name.decode() == rt["name"], key
        assert (fd.mfp, fd.beta) == (rt["fd"][0], rt["fd"][1]), key
        if mode == "UNC" and th == 1:
            fn = {16: lib.test_gaxtuh1hw16w, 8: lib.test_gaxtuh1hw08w, 4: lib.test_gaxtuh1hw04w}
            res = fn.get(thw, lib.test_gaxtuh1hw16w)(128, 256, t, R.f64p(y_ref))
        elif mode == "UNC":
            res = lib.test_gaxtuh(2, 256, t, R.f64p(y_ref))
        elif th == 1:
            res = lib.test_gaxtch1(bs, t, R.f64p(y_ref))
        else:
            res = lib.test_gaxtch(256, t, R.f64p(y_ref))
        check(res, key)
        R.free_struct_arrays(t, ("ax", "sec", "con"))
