"""The reference's own GPU products (gcsr, gk1, gaxc, gaxtuh, gaxtuh1hw16w, gaxtch1, gaxtch
from cudaSpmv.cu:531-2285, compiled unchanged for sm_100a into oracle/_ref) beside the engine's
drop-in entry points of the same names, on the same matrices and x (x baked into the AXC /
AXT layouts, as the reference's converters do).  Both meet the reference's own error check
against its CPU ncsr; on the power-law matrix the engine's K1 product takes less device time
than the reference's gk1 on the same GPU.  Matrices here have no empty rows: the reference's gk1 reads a chunk's first
slot unconditionally (cudaSpmv.cu:861)."""
import ctypes as C
import statistics

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _matrices():
    from gpu_spmv_b200 import matgen

    yield "laplacian_512", matgen.laplacian2d(512)
    yield "powerlaw_256k", matgen.powerlaw(nrows=262144, nnz=4194304, seed=1)


@pytest.mark.parametrize("which", [0, 1], ids=["laplacian_512", "powerlaw_256k"])
def test_reference_gpu_products_beside_dropin(ref, port, which):
    import torch

    from gpu_spmv_b200 import _lib as L
    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import refapi as R
    from gpu_spmv_b200 import matgen

    name, (row, col, val) = list(_matrices())[which]
    n = len(row) - 1
    assert np.all(np.diff(row.astype(np.int64)) > 0)
    x = matgen.vector(n, "uniform", -1.0, 1.0, seed=0)
    y_ref = ref.ncsr(row, col, val, x)
    _, mag = port.csr_truth(row, col, val, x)
    tol = 1e-13 * float(mag.max())

    theirs = ref.gpu_products(row, col, val, x, y_ref, reps=3)
    for k, v in theirs.items():
        assert v["seconds"] > 0 and v["aErr"] <= tol, (k, v)

    lib = L.lib()
    lib.gs_set_num_ite(20)
    try:
        h = R.csr_struct(row, col, val, name=name + ".bin")
        ours = {}
        res = lib.test_gcsr(256, h.s, R.f64p(x), R.f64p(y_ref))
        ours["gcsr"] = res
        k1 = L.StrMatK1()
        lib.getFormatDataK1(32, h.s, R.f64p(x), C.byref(k1))
        ours["gk1"] = lib.test_gk1(256, k1, R.f64p(x), R.f64p(y_ref))
        R.free_struct_arrays(k1, ("permi", "nmc", "chp", "val", "col"))
        a = L.StrMatAXC()
        lib.getFormatDataAXC(1, 32, h.s, R.f64p(x), C.byref(a))
        ours["gaxc"] = lib.test_gaxc(256, a, R.f64p(y_ref))
        R.free_struct_arrays(a, ("ax", "brp", "mapx"))
        for mode, thw, th, key, fn in (
                (b"UNC", 32, 4, "gaxtuh4", lambda t: lib.test_gaxtuh(4, 256, t, R.f64p(y_ref))),
                (b"UNC", 16, 1, "gaxtuh1hw16",
                 lambda t: lib.test_gaxtuh1hw16w(128, 256, t, R.f64p(y_ref))),
                (b"COM", 32, 1, "gaxtch1", lambda t: lib.test_gaxtch1(256, t, R.f64p(y_ref))),
                (b"COM", 32, 4, "gaxtch4", lambda t: lib.test_gaxtch(256, t, R.f64p(y_ref)))):
            t = L.StrMatAXT()
            lib.getFormatDataAXT(1, 256, thw, th, mode, h.s, R.f64p(x), C.byref(t))
            ours[key] = fn(t)
            R.free_struct_arrays(t, ("ax", "sec", "con"))
    finally:
        lib.gs_set_num_ite(250)
    for k, r in ours.items():
        assert r.et > 0 and r.sErr.aErr <= tol, (k, bytes(r.name), r.sErr.aErr)

    # the engine's K1 product against the reference's gk1 on the same GPU: device time per
    # launch over 20 launches back to back (the reference times one launch after its copies)
    A = E.Matrix(row, col, val, ncols=n, fmt="K1")
    dx = torch.from_numpy(x).cuda()
    y = A.spmv(dx)
    ts = []
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(20):
            A.spmv(dx, y)
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) * 1e-3 / 20)
    A.close()
    ours_k1 = statistics.median(ts)
    print(name, {k: round(v["seconds"] * 1e6, 1) for k, v in theirs.items()},
          {k: round(r.et * 1e6, 1) for k, r in ours.items()}, "K1", round(ours_k1 * 1e6, 1))
    # timed against each other only where the product streams from HBM: the Laplacian sits
    # in L2, where both take about 10 us and the reference's single timed launch varies by 2x
    if which == 1:
        assert ours_k1 < theirs["gk1"]["seconds"]
