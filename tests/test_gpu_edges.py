"""Edge shapes on the GPU, every format: matrices with no stored element, one row, rows
not a multiple of 32, wide and tall shapes, runs of empty rows and a few very long rows,
over seeded random instances.  FP64 products meet max|y - y_ref| <= 1e-13 (|A||x|)_i against
the oracle's CPU loop; FP32 storage meets its per-row bound; multi-RHS products and the
adjoint match the explicit transpose."""
import numpy as np
import pytest
import torch

from mats import csr_from_lengths, within_bound

pytestmark = pytest.mark.gpu

FORMATS = [dict(fmt="CSR"), dict(fmt="K1"), dict(fmt="AXC", hbs=32), dict(fmt="AXC", hbs=8),
           dict(fmt="AXT", mode="UNC", tileH=1, tileHW=4),
           dict(fmt="AXT", mode="UNC", tileH=1, tileHW=32),
           dict(fmt="AXT", mode="UNC", tileH=4, tileHW=32),
           dict(fmt="AXT", mode="UNC", tileH=16, tileHW=32),
           dict(fmt="AXT", mode="COM", tileH=1, tileHW=32, bs=64),
           dict(fmt="AXT", mode="COM", tileH=8, tileHW=32)]


def _shape(kind, rng):
    if kind == "no_elements":
        n = 45
        return np.zeros(n + 1, np.uint32), np.zeros(0, np.uint32), np.zeros(0), n
    if kind == "one_empty_row":
        return np.zeros(2, np.uint32), np.zeros(0, np.uint32), np.zeros(0), 7
    if kind == "one_full_row":
        row, col, val = csr_from_lengths([300], 300, rng)
        return row, col, val, 300
    if kind == "wide":  # 33 rows, 5000 columns
        row, col, val = csr_from_lengths(rng.integers(0, 200, 33), 5000, rng)
        return row, col, val, 5000
    if kind == "tall":  # 3001 rows, 20 columns
        row, col, val = csr_from_lengths(rng.integers(0, 21, 3001), 20, rng)
        return row, col, val, 20
    if kind == "empty_runs":
        n = 1000
        lens = rng.integers(0, 9, n)
        lens[100:400] = 0
        lens[-65:] = 0
        row, col, val = csr_from_lengths(lens, n, rng)
        return row, col, val, n
    if kind == "long_rows":
        n = 777
        lens = rng.integers(0, 4, n)
        lens[rng.choice(n, 5, replace=False)] = rng.integers(600, 777, 5)
        row, col, val = csr_from_lengths(lens, n, rng)
        return row, col, val, n
    raise KeyError(kind)


KINDS = ["no_elements", "one_empty_row", "one_full_row", "wide", "tall", "empty_runs",
         "long_rows"]


def _ids(f):
    return "_".join(f"{k}{v}" for k, v in f.items())


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("fmt", FORMATS, ids=[_ids(f) for f in FORMATS])
def test_edge_shapes_fp64(port, kind, fmt):
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(sum(map(ord, kind)) + 3)
    row, col, val, ncols = _shape(kind, rng)
    n = len(row) - 1
    A = E.Matrix(row, col, val, ncols=ncols, **fmt)
    x = rng.uniform(-1, 1, ncols)
    y = A.spmv(torch.from_numpy(x).cuda()).cpu().numpy()
    assert y.shape == (n,)
    _, mag = port.csr_truth(row, col, val, x)
    assert within_bound(y, port.csr_spmv(row, col, val, x), mag)
    assert np.all(y[np.diff(row) == 0] == 0)  # empty rows are written, as zero
    A.close()


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("fmt", [dict(fmt="K1"), dict(fmt="CSR"),
                                 dict(fmt="AXT", mode="UNC", tileH=1, tileHW=8)],
                         ids=["k1", "csr", "unc1hw8"])
@pytest.mark.parametrize("itype", ["u32", "u16"])
def test_edge_shapes_fp32(port, kind, fmt, itype):
    from gpu_spmv_b200 import GSError
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(sum(map(ord, kind)) + 4)
    row, col, val, ncols = _shape(kind, rng)
    try:
        A = E.Matrix(row, col, val, ncols=ncols, vtype="f32", itype=itype, **fmt)
    except GSError as e:  # 16-bit offsets that do not fit are refused, never truncated
        assert itype == "u16" and "16-bit" in str(e)
        return
    x = rng.uniform(-1, 1, ncols)
    y = A.spmv(torch.from_numpy(x).float().cuda()).double().cpu().numpy()
    exact, mag = port.csr_truth(row, col, val, x)
    lens = np.diff(row).astype(np.float64)
    assert np.all(np.abs(y - exact) <= 2.0 ** -24 * (3 + lens) * mag)
    A.close()


@pytest.mark.parametrize("kind", ["no_elements", "one_full_row", "empty_runs", "long_rows"])
def test_edge_shapes_spmm_adjoint(port, kind):
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(sum(map(ord, kind)) + 5)
    row, col, val, ncols = _shape(kind, rng)
    n = len(row) - 1
    A = E.Matrix(row, col, val, ncols=ncols, fmt="K1", adjoint=True)
    X = torch.from_numpy(rng.uniform(-1, 1, (ncols, 5))).cuda()
    Y = A.spmm(X)
    for r in range(5):
        assert torch.equal(Y[:, r], A.spmv(X[:, r].contiguous()))
    Yb = rng.standard_normal((n, 5))
    Xb, vb = A.adjoint(torch.from_numpy(Yb).cuda(), X)
    rows = np.repeat(np.arange(n), np.diff(row))
    for r in range(5):
        ref = np.zeros(ncols)
        np.add.at(ref, col, val * Yb[rows, r])
        mag = np.zeros(ncols)
        np.add.at(mag, col, np.abs(val * Yb[rows, r]))
        assert np.all(np.abs(Xb[:, r].cpu().numpy() - ref) <= 1e-13 * mag + 1e-300)
    Xh = X.cpu().numpy()
    vref = np.einsum("ek,ek->e", Yb[rows], Xh[col]) if len(col) else np.zeros(0)
    vmag = np.einsum("ek,ek->e", np.abs(Yb[rows]), np.abs(Xh[col])) if len(col) else vref
    assert np.all(np.abs(vb.cpu().numpy() - vref) <= 1e-13 * vmag + 1e-300)
    A.close()
