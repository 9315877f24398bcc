"""Parity at the benchmark sizes: the power-law matrix (4,194,304 rows, 67,108,864 nnz),
the 27-point stencil 160^3 (109,215,352 nnz) and the 512^2 Laplacian, each product
checked row by row against the oracle's CPU loop (the restated ncsr) on the same inputs:
FP64 within 1e-13 (|A||x|)_i, FP32 values with 16-bit steps within
(2^-24 (3 + len_i)) (|A||x|)_i.  Plus a size-independent property: linearity,
A(2x - y) = 2Ax - Ay, on the same kernels."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def powerlaw():
    from gpu_spmv_b200 import matgen

    row, col, val = matgen.powerlaw(seed=1)
    x = matgen.vector(len(row) - 1, "uniform", -1.0, 1.0, seed=1001)
    return row, col, val, x


def _check(port, row, col, val, x, y, rel=1e-13):
    ref = port.csr_spmv(row, col, val, x)
    _, mag = port.csr_truth(row, col, val, x)
    err = np.abs(y - ref)
    assert np.all(err <= rel * mag), float(np.max(err / np.maximum(mag, 1e-300)))


@pytest.mark.parametrize("fmt", [dict(fmt="K1"), dict(fmt="AXT", mode="UNC", tileH=4, tileHW=32),
                                 dict(fmt="CSR")], ids=["k1", "unc4", "csr"])
def test_powerlaw_64M(port, powerlaw, fmt):
    from gpu_spmv_b200 import engine as E

    row, col, val, x = powerlaw
    n = len(row) - 1
    assert len(col) == 67108864 and n == 4194304
    A = E.Matrix(row, col, val, ncols=n, **fmt)
    dx = torch.from_numpy(x).cuda()
    y = A.spmv(dx).cpu().numpy()
    _check(port, row, col, val, x, y)
    # linearity with a second vector
    x2 = np.random.default_rng(5).uniform(-1, 1, n)
    y2 = A.spmv(torch.from_numpy(x2).cuda()).cpu().numpy()
    y3 = A.spmv(torch.from_numpy(2 * x - x2).cuda()).cpu().numpy()
    _, m1 = port.csr_truth(row, col, val, x)
    _, m2 = port.csr_truth(row, col, val, x2)
    assert np.all(np.abs(y3 - (2 * y - y2)) <= 4e-13 * (2 * m1 + m2))
    A.close()


def test_stencil27_160(port):
    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import matgen

    row, col, val = matgen.stencil27(160, seed=2)
    n = len(row) - 1
    assert len(col) == 109215352
    x = matgen.vector(n, "normal", seed=2)
    A = E.Matrix(row, col, val, ncols=n, fmt="K1")
    y = A.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
    _check(port, row, col, val, x, y)
    A.close()
    B = E.Matrix(row, col, val, ncols=n, fmt="K1", vtype="f32", itype="u16")
    y = B.spmv(torch.from_numpy(x).float().cuda()).double().cpu().numpy()
    exact, mag = port.csr_truth(row, col, val, x)
    lens = np.diff(row).astype(np.float64)
    assert np.all(np.abs(y - exact) <= 2.0 ** -24 * (3 + lens) * mag)
    assert np.max(np.abs(y - exact) / mag) < 1e-6
    B.close()


def test_laplacian_512(port):
    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import matgen

    row, col, val = matgen.laplacian2d(512)
    n = len(row) - 1
    assert n == 262144 and len(col) == 1308672
    x = matgen.vector(n, "uniform", -1.0, 1.0, seed=0)
    for kw in (dict(fmt="CSR"), dict(fmt="AXT", mode="COM", tileH=1, tileHW=32),
               dict(fmt="AXT", mode="UNC", tileH=1, tileHW=16), dict(fmt="K1")):
        A = E.Matrix(row, col, val, ncols=n, **kw)
        y = A.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
        _check(port, row, col, val, x, y)
        # K1: each row summed by one lane in slot (= CSR) order: the CPU loop's bits
        if kw["fmt"] == "K1":
            assert np.array_equal(y, port.csr_spmv(row, col, val, x))
        A.close()


@pytest.mark.parametrize("fmt", [dict(fmt="K1"),
                                 dict(fmt="AXT", mode="UNC", tileH=4, tileHW=32),
                                 dict(fmt="AXT", mode="COM", tileH=1, tileHW=32, bs=256)],
                         ids=["k1", "unc4", "com1"])
def test_powerlaw_64M_conversion_bit_exact(port, powerlaw, fmt):
    """The device converters on the headline matrix (4,194,304 rows, 67,108,864 nnz)
    against the oracle's restated converters, which the CPU suite pins to the reference's
    own at this size: K1 permi / nmc / chp / val / col (the stable length sort of 4M rows
    with heavy ties, cudaSpmv.cu:716-846), AXT sec / con and the value and column slots
    (cudaSpmv.cu:1158-1566), bit for bit."""
    from gpu_spmv_b200 import engine as E

    row, col, val, x = powerlaw
    n = len(row) - 1
    A = E.Matrix(row, col, val, ncols=n, keep_layout=True, **fmt)
    lay = A.layout()
    i = A.info
    if fmt["fmt"] == "K1":
        k = port.k1(row, col, val)
        assert (i.chunkNum, i.lenVC) == (k["chunkNum"], k["lenVC"])
        for key in ("permi", "nmc", "chp", "val", "col"):
            assert np.array_equal(lay[key], k[key]), key
    else:
        t = port.axt(row, col, val, fmt["tileHW"], fmt["tileH"], fmt["mode"],
                     bs=fmt.get("bs", 256))
        d = t["dims"]
        assert (i.tileN, i.lenAX, i.lenSEC, i.lenCON, i.log, i.logTH) == \
            (d.tileN, d.lenAX, d.lenSEC, d.lenCON, d.log, d.logTH)
        for key in ("val", "col", "sec", "con"):
            assert np.array_equal(lay[key], t[key]), key
    del lay
    # and the product from the converted layout
    _check(port, row, col, val, x, A.spmv(torch.from_numpy(x).cuda()).cpu().numpy())
    A.close()


@pytest.mark.parametrize("fmt", [dict(fmt="AXT", mode="UNC", tileH=8, tileHW=32),
                                 dict(fmt="AXT", mode="COM", tileH=8, tileHW=32, bs=256),
                                 dict(fmt="AXC", hbs=32),
                                 dict(fmt="AXT", mode="UNC", tileH=1, tileHW=4)],
                         ids=["unc8", "com8", "axc", "unc1hw4"])
def test_powerlaw_64M_other_formats(port, powerlaw, fmt):
    """Row-stream layouts with 8 positions per lane and ~2048-position warp ranges, and the
    tile kernel, on the full power-law matrix: within 1e-13 (|A||x|)_i of the oracle."""
    from gpu_spmv_b200 import engine as E

    row, col, val, x = powerlaw
    n = len(row) - 1
    A = E.Matrix(row, col, val, ncols=n, **fmt)
    _check(port, row, col, val, x, A.spmv(torch.from_numpy(x).cuda()).cpu().numpy())
    A.close()


def test_stencil27_160_row_stream(port):
    """CSR (8 positions per lane: the stencil's columns are local) and AXT COM tileH 1 on
    the 27-point stencil 160^3 against the oracle."""
    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import matgen

    row, col, val = matgen.stencil27(160, seed=2)
    n = len(row) - 1
    x = matgen.vector(n, "normal", seed=2)
    for kw in (dict(fmt="CSR"), dict(fmt="AXT", mode="COM", tileH=1, tileHW=32),
               dict(fmt="AXT", mode="UNC", tileH=4, tileHW=32)):
        A = E.Matrix(row, col, val, ncols=n, **kw)
        if kw["fmt"] == "CSR":
            assert A.info.lane_positions == 8
        _check(port, row, col, val, x, A.spmv(torch.from_numpy(x).cuda()).cpu().numpy())
        A.close()


@pytest.mark.parametrize("th", [2, 4])
def test_grouped_tiles_random_rows(port, th):
    """UNC layouts of 32-wide tiles, tileH 2 and 4, on a matrix with random columns (the
    row-stream kernel then takes the tiles a warp owns two at a time): 1.5M rows of 0-40
    elements (empty rows included) and 16 rows of 20k-200k elements that cross many tiles
    and warp ranges, within 1e-13 (|A||x|)_i of the oracle; the 27-point stencil's local
    columns keep one tile per step."""
    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import matgen

    rng = np.random.default_rng(11)
    n = 1_500_000
    lens = rng.integers(0, 41, n)
    lens[rng.choice(n, 16, replace=False)] = rng.integers(20_000, 200_000, 16)
    row = np.zeros(n + 1, dtype=np.uint32)
    row[1:] = np.cumsum(lens)
    nnz = int(row[-1])
    col = rng.integers(0, n, nnz, dtype=np.uint32)
    val = rng.uniform(-1.0, 1.0, nnz)
    x = rng.uniform(-1.0, 1.0, n)
    A = E.Matrix(row, col, val, ncols=n, fmt="AXT", mode="UNC", tileH=th, tileHW=32)
    assert A.info.tiles_per_step == 2
    _check(port, row, col, val, x, A.spmv(torch.from_numpy(x).cuda()).cpu().numpy())
    A.close()
    srow, scol, sval = matgen.stencil27(40, seed=2)
    S = E.Matrix(srow, scol, sval, ncols=len(srow) - 1, fmt="AXT", mode="UNC", tileH=th,
                 tileHW=32)
    assert S.info.tiles_per_step == 1
    sx = matgen.vector(len(srow) - 1, "normal", seed=2)
    _check(port, srow, scol, sval, sx, S.spmv(torch.from_numpy(sx).cuda()).cpu().numpy())
    S.close()
