"""Native layer on the GPU against the CPU oracle: every format's device converter output is
bit-identical to the restated reference converter, and every format's SpMV matches the
reference's CPU CSR path within max|y - y_ref| <= 1e-13 * (|A||x|)_i (FP64)."""
import numpy as np
import pytest
import torch

from mats import AXT_PARAMS, CASES, case, within_bound

pytestmark = pytest.mark.gpu

# beyond the reference's parameter sets: tileH 2 (its own 2-wide kernel), 3 and 5 (tile
# columns shorter than the kernel's lane width)
EXTRA_AXT = [("COM", 2, 32, 256), ("COM", 3, 32, 256), ("COM", 5, 32, 256), ("UNC", 3, 32, 256)]
FORMATS = [("CSR", {}), ("K1", {}), ("AXC", {"hbs": 32}), ("AXC", {"hbs": 16})] + [
    ("AXT", {"mode": m, "tileH": th, "tileHW": thw, "bs": bs})
    for (m, th, thw, bs) in AXT_PARAMS + EXTRA_AXT]


def _ids(p):
    f, kw = p
    return f + "".join(f"_{k}{v}" for k, v in kw.items())


def _square_ncols(row, col):
    n = len(row) - 1
    return max(n, int(col.max()) + 1 if len(col) else n)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("fmt", FORMATS, ids=[_ids(p) for p in FORMATS])
def test_native_layout_and_spmv(port, name, fmt):
    from gpu_spmv_b200 import engine as E

    f, kw = fmt
    rng = np.random.default_rng(sum(map(ord, name)) + 17)
    row, col, val = case(name, rng)
    ncols = _square_ncols(row, col)
    A = E.Matrix(row, col, val, ncols=ncols, fmt=f, keep_layout=True, **kw)
    lay = A.layout()
    i = A.info
    if f == "CSR":
        assert np.array_equal(lay["val"], val) and np.array_equal(lay["col"], col)
        assert np.array_equal(lay["rpos"], row)
    elif f == "K1":
        k = port.k1(row, col, val)
        for key in ("permi", "nmc", "chp", "val", "col"):
            assert np.array_equal(lay[key], k[key]), key
        assert i.lenVC == k["lenVC"] and i.chunkNum == k["chunkNum"]
    elif f == "AXC":
        a = port.axc(row, col, val, hbs=kw["hbs"])
        assert i.lenAX == a["lenAX"]
        for key in ("brp", "mapx", "val", "col"):
            assert np.array_equal(lay[key], a[key]), key
    else:
        t = port.axt(row, col, val, kw["tileHW"], kw["tileH"], kw["mode"], bs=kw["bs"])
        d = t["dims"]
        assert (i.tileN, i.lenAX, i.lenSEC, i.lenCON, i.log, i.logTH) == \
            (d.tileN, d.lenAX, d.lenSEC, d.lenCON, d.log, d.logTH)
        for key in ("val", "col", "sec", "con"):
            assert np.array_equal(lay[key], t[key]), key
    x = rng.uniform(-1, 1, ncols)
    y = A.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
    y_ref = port.csr_spmv(row, col, val, x)  # the reference's CPU path (ncsr)
    _, mag = port.csr_truth(row, col, val, x)
    assert within_bound(y, y_ref, mag), np.max(np.abs(y - y_ref) / np.maximum(mag, 1e-300))
    # deterministic: a second launch gives the same bits
    y2 = A.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
    assert np.array_equal(y, y2)
    A.close()


@pytest.mark.parametrize("name", ["mixed", "row0_empty", "dense_row", "powerlaw_small"])
@pytest.mark.parametrize("mode,th", [("COM", 4), ("COM", 8), ("COM", 16), ("UNC", 4),
                                     ("UNC", 8), ("UNC", 16)])
def test_tma_staging_matches_plain_loads(port, name, mode, th):
    """32-wide tiled layouts run on the TMA-staged kernel; the plain-load kernel sums in the
    same order, so the two agree to the last bit, and no bounded wait timed out."""
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(th + len(name))
    row, col, val = case(name, rng)
    n = len(row) - 1
    ncols = _square_ncols(row, col)
    A = E.Matrix(row, col, val, ncols=ncols, fmt="AXT", mode=mode, tileH=th, tileHW=32)
    x = torch.from_numpy(rng.uniform(-1, 1, ncols)).cuda()
    y_tma = A.spmv(x, tma=True).cpu().numpy()
    y_ldg = A.spmv(x, tma=False).cpu().numpy()
    assert A.device_status() == 0
    assert np.array_equal(y_tma, y_ldg)
    _, mag = port.csr_truth(row, col, val, x.cpu().numpy())
    assert within_bound(y_tma, port.csr_spmv(row, col, val, x.cpu().numpy()), mag)
    assert len(y_tma) == n


@pytest.mark.parametrize("name", ["mixed", "row0_empty", "dense_row", "laplacian"])
@pytest.mark.parametrize("fmt", [dict(fmt="CSR"), dict(fmt="AXC", hbs=32),
                                 dict(fmt="AXT", mode="UNC", tileH=1, tileHW=4),
                                 dict(fmt="AXT", mode="COM", tileH=1, tileHW=32)],
                         ids=["csr", "axc", "unc1hw4", "com1"])
def test_striped_variant(port, name, fmt):
    """The striped (one position per lane per chunk) kernel variant meets the same bound."""
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(7 + len(name))
    row, col, val = case(name, rng)
    ncols = _square_ncols(row, col)
    A = E.Matrix(row, col, val, ncols=ncols, **fmt)
    xh = rng.uniform(-1, 1, ncols)
    y = A.spmv(torch.from_numpy(xh).cuda(), striped=True).cpu().numpy()
    _, mag = port.csr_truth(row, col, val, xh)
    assert within_bound(y, port.csr_spmv(row, col, val, xh), mag)


@pytest.mark.parametrize("name", ["mixed", "laplacian", "powerlaw_small"])
def test_csr_from_device_arrays(port, name):
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(5)
    row, col, val = case(name, rng)
    n = len(row) - 1
    x = rng.uniform(-1, 1, n)
    dev = torch.device("cuda")
    y = E.csr_spmv_f64(E.to_device_u32(row, dev), E.to_device_u32(col, dev),
                       torch.from_numpy(val).cuda(), torch.from_numpy(x).cuda())
    y = y.cpu().numpy()
    y_ref = port.csr_spmv(row, col, val, x)
    _, mag = port.csr_truth(row, col, val, x)
    assert within_bound(y, y_ref, mag)
    # rows that one lane sums alone reproduce the CPU loop bit for bit
    short = np.diff(row) <= 1
    assert np.array_equal(y[short], y_ref[short])


def test_invalid_csr_rejected():
    from gpu_spmv_b200 import GSError
    from gpu_spmv_b200 import engine as E

    row = np.array([0, 2, 1, 3], np.uint32)  # not monotone
    col = np.array([0, 1, 2], np.uint32)
    val = np.ones(3)
    with pytest.raises(GSError, match="GS_ERR_INVALID"):
        E.Matrix(row, col, val, fmt="CSR")
    row = np.array([0, 1, 2, 3], np.uint32)
    col = np.array([0, 1, 7], np.uint32)  # column out of range
    with pytest.raises(GSError, match="ncols"):
        E.Matrix(row, col, val, fmt="AXT", mode="UNC", tileH=1, tileHW=4)


def test_com_header_overflow_reported():
    """row << log must fit 32 bits (cudaSpmv.cu:1338 packs it silently): with log = 10
    (bs = 1024) a matrix of more than 2^22 rows cannot be stored in the COM layout."""
    from gpu_spmv_b200 import GSError
    from gpu_spmv_b200 import engine as E

    n = (1 << 22) + 2
    row = np.arange(n + 1, dtype=np.uint32)
    col = np.arange(n, dtype=np.uint32)
    val = np.ones(n)
    with pytest.raises(GSError, match="GS_ERR_OVERFLOW"):
        E.Matrix(row, col, val, fmt="AXT", mode="COM", tileH=1, tileHW=32, bs=1024,
                 keep_layout=True)
    # without the reference metadata the native layout needs no header and converts
    A = E.Matrix(row, col, val, fmt="AXT", mode="COM", tileH=1, tileHW=32, bs=1024)
    x = torch.arange(n, dtype=torch.float64, device="cuda")
    assert torch.equal(A.spmv(x), x)


@pytest.mark.parametrize("fmt,vtype", [("K1", "f64"), ("CSR", "f64"), ("K1", "f32")])
def test_host_stream_products(port, fmt, vtype):
    """gs_spmv_host_stream: each of several host vectors copied in, multiplied and copied
    out, overlapped across vectors; every y_k equals the device product of x_k."""
    import ctypes as C

    from gpu_spmv_b200 import _lib as L
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(8)
    row, col, val = case("powerlaw_small", rng)
    n = len(row) - 1
    A = E.Matrix(row, col, val, ncols=n, fmt=fmt, vtype=vtype)
    dt = torch.float64 if vtype == "f64" else torch.float32
    code = L.GS_F64 if vtype == "f64" else L.GS_F32
    k = 7
    X = torch.from_numpy(rng.uniform(-1, 1, (k, n))).to(dt).pin_memory()
    Y = torch.empty(k, n, dtype=dt).pin_memory()
    L.check(L.lib().gs_spmv_host_stream(A._h, X.data_ptr(), n, code, Y.data_ptr(), n, code, k,
                                        0, E.stream_handle()), "stream")
    for i in range(k):
        assert torch.equal(Y[i], A.spmv(X[i].cuda()).cpu()), i
    # stride 0: the same vector every time, the last y stays
    L.check(L.lib().gs_spmv_host_stream(A._h, X.data_ptr(), 0, code, Y.data_ptr(), 0, code, 3,
                                        0, E.stream_handle()), "stream")
    assert torch.equal(Y[0], A.spmv(X[0].cuda()).cpu())
    A.close()


def test_create_from_host_arrays(port):
    """gs_matrix_create_host: the same matrix as from device arrays, from host CSR arrays."""
    import ctypes as C

    from gpu_spmv_b200 import _lib as L
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(12)
    row, col, val = case("powerlaw_small", rng)
    n = len(row) - 1
    row = np.ascontiguousarray(row, np.uint32)
    col = np.ascontiguousarray(col, np.uint32)
    val = np.ascontiguousarray(val, np.float64)
    p = L.ConvertParams(L.GS_FMT_AXT, 32, 4, 256, L.GS_AXT_UNC, 32, L.GS_F64, L.GS_IDX_U32, 0)
    h = C.c_void_p()
    L.check(L.lib().gs_matrix_create_host(C.byref(h), C.byref(p), n, n, len(col),
                                          row.ctypes.data, col.ctypes.data, val.ctypes.data,
                                          L.GS_F64, None), "create_host")
    x = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    L.check(L.lib().gs_spmv(h, x.data_ptr(), L.GS_F64, y.data_ptr(), L.GS_F64, 0, None), "spmv")
    A = E.Matrix(row, col, val, ncols=n, fmt="AXT", mode="UNC", tileH=4, tileHW=32)
    assert torch.equal(y, A.spmv(x))
    L.lib().gs_matrix_destroy(h)


def _lane_case(kind):
    from gpu_spmv_b200 import matgen

    if kind == "random":  # 10-40 uniformly random columns per row: gather-bound
        rng = np.random.default_rng(11)
        from mats import csr_from_lengths
        return csr_from_lengths(rng.integers(10, 41, 6000), 6000, rng)
    if kind == "banded":  # 20-40 columns in a band of 129: local columns
        return matgen.banded(20000, 64, 20, 40, seed=12)
    return matgen.laplacian2d(96)  # 5 per row


@pytest.mark.parametrize("kind,expect", [("random", 4), ("banded", 8), ("short", 4)])
@pytest.mark.parametrize("fmt", [dict(fmt="CSR"), dict(fmt="AXT", mode="COM", tileH=1, tileHW=32)],
                         ids=["csr", "com1"])
def test_lane_positions_choice(port, kind, expect, fmt):
    """FP64 CSR / COM tileH=1 products take 4 positions per lane when their x gathers are
    random or their rows short, 8 when rows of local columns stream; both meet the bound,
    and so does the device-array CSR entry point, which makes the same choice per call."""
    from gpu_spmv_b200 import engine as E

    row, col, val = _lane_case(kind)
    n = len(row) - 1
    A = E.Matrix(row, col, val, ncols=n, **fmt)
    assert A._info().lane_positions == expect
    x = np.random.default_rng(3).uniform(-1, 1, n)
    y_ref = port.csr_spmv(row, col, val, x)
    _, mag = port.csr_truth(row, col, val, x)
    assert within_bound(A.spmv(torch.from_numpy(x).cuda()).cpu().numpy(), y_ref, mag)
    assert within_bound(A.spmv(torch.from_numpy(x).cuda(), striped=True).cpu().numpy(), y_ref,
                        mag)
    A.close()
    dev = torch.device("cuda")
    y = E.csr_spmv_f64(E.to_device_u32(row, dev), E.to_device_u32(col, dev),
                       torch.from_numpy(val).cuda(), torch.from_numpy(x).cuda())
    assert within_bound(y.cpu().numpy(), y_ref, mag)


@pytest.mark.parametrize("kind,expect", [("random", 4), ("banded", 8)])
@pytest.mark.parametrize("fmt", [dict(fmt="AXC", hbs=32),
                                 dict(fmt="AXT", mode="UNC", tileH=1, tileHW=32)],
                         ids=["axc32", "unc1hw32"])
def test_lane_positions_padded32(port, kind, expect, fmt):
    """Layouts whose rows are padded to 32 positions (AXC hbs 32, UNC tileH 1 tileHW 32)
    take 4 positions per lane when their x gathers are random, 8 when the columns are local;
    both within the FP64 bound of the oracle."""
    from gpu_spmv_b200 import engine as E

    row, col, val = _lane_case(kind)
    n = len(row) - 1
    A = E.Matrix(row, col, val, ncols=n, **fmt)
    assert A._info().lane_positions == expect
    x = np.random.default_rng(4).uniform(-1, 1, n)
    y_ref = port.csr_spmv(row, col, val, x)
    _, mag = port.csr_truth(row, col, val, x)
    assert within_bound(A.spmv(torch.from_numpy(x).cuda()).cpu().numpy(), y_ref, mag)
    A.close()


@pytest.mark.parametrize("fmt", [dict(fmt="CSR"), dict(fmt="CSR", vtype="f32"),
                                 dict(fmt="AXT", mode="COM", tileH=1, tileHW=32),
                                 dict(fmt="AXT", mode="COM", tileH=2, tileHW=32),
                                 dict(fmt="AXT", mode="COM", tileH=4, tileHW=32),
                                 dict(fmt="AXT", mode="COM", tileH=6, tileHW=32),
                                 dict(fmt="AXT", mode="UNC", tileH=6, tileHW=32)],
                         ids=["csr", "csr-f32", "com1", "com2", "com4", "com6", "unc6"])
def test_rows_across_warp_ranges(port, fmt):
    """Rows much longer than a warp's range of windows (up to 70,000 elements, next to empty
    and one-element rows; the warp where a row starts sums it past its range end): the bound
    holds and repeated products are bit-identical."""
    from gpu_spmv_b200 import engine as E
    from mats import csr_from_lengths

    rng = np.random.default_rng(21)
    lens = rng.integers(0, 9, 4000)
    for i, L in ((0, 70000), (1, 1), (2, 4095), (3, 0), (4, 33000), (900, 1024), (901, 2048),
                 (2000, 50000), (3999, 12345)):
        lens[i] = L
    row, col, val = csr_from_lengths(lens, 200000, rng)
    A = E.Matrix(row, col, val, ncols=200000, **fmt)
    f32 = fmt.get("vtype") == "f32"
    x = rng.uniform(-1, 1, 200000)
    xd = torch.from_numpy(x).cuda()
    if f32:
        xd = xd.float()
    y1 = A.spmv(xd)
    y2 = A.spmv(xd)
    assert torch.equal(y1, y2)
    y = y1.double().cpu().numpy()
    exact, mag = port.csr_truth(row, col, val, x.astype(np.float32).astype(np.float64) if f32 else x)
    if f32:
        lensf = np.diff(row).astype(np.float64)
        vals32 = val.astype(np.float32).astype(np.float64)
        e32, m32 = port.csr_truth(row, col, vals32, x.astype(np.float32).astype(np.float64))
        assert np.all(np.abs(y - e32) <= 2.0 ** -24 * (3 + lensf) * m32 + 1e-30)
    else:
        assert within_bound(y, port.csr_spmv(row, col, val, x), mag)
    A.close()
