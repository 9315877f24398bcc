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
