"""FP32 multi-RHS, batched and differentiable products against the oracle's CPU loop.

The FP32 kernels (k_k1_mm<float, K>, the batch kernels k_batch / k_batch_band and the
transposed-K1 adjoint) store values and right-hand sides in FP32 and form products and sums
in FP32.  Each column is checked against the oracle's CPU CSR loop (the restated ncsr,
cudaSpmv.cu:451-466) run in FP64 on the same FP32 numbers, row by row:

    |y_i - y64_i| <= 2^-24 (3 + len_i) (|A||x|)_i

(len_i products and sums, each rounded once to FP32).  At the sizes of the benchmark's
batched configuration (256 banded matrices, seed 3) and differentiable configuration
(power-law 1,048,576 rows, 16,777,216 nnz, 8 right-hand sides, seed 4) the largest relative
error is also held to the stated 1e-6 of (|A||x|)_i, and the differentiable configuration's
gradients are checked in FP64 against central finite differences on 64 entries."""
import numpy as np
import pytest
import torch

from mats import case

pytestmark = pytest.mark.gpu

U = 2.0 ** -24


def _fp32_bound_ok(Y, A64, Xs64, row, col, port):
    """Every column of Y (FP32, [n, k]) within the FP32 bound of the FP64 oracle product of
    A64 (the FP32 values as FP64) and Xs64; returns the largest error / (|A||x|)_i."""
    lens = np.diff(row).astype(np.float64)
    ref = port.csr_spmm(row, col, A64, Xs64)
    mag = port.csr_spmm(row, col, np.abs(A64), np.abs(Xs64))
    err = np.abs(Y.astype(np.float64) - ref)
    assert np.all(err <= U * (3.0 + lens)[:, None] * mag + 1e-300), \
        float(np.max(err / np.maximum(mag, 1e-300)))
    return float(np.max(err / np.maximum(mag, 1e-300)))


@pytest.mark.parametrize("name", ["mixed", "row0_empty", "dense_row", "powerlaw_small",
                                  "laplacian", "k1_empty_chunk"])
@pytest.mark.parametrize("k", [1, 2, 4, 8, 16, 32])
def test_fp32_spmm_columns_against_oracle(port, name, k):
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(sum(map(ord, name)) + 7 * k)
    row, col, val = case(name, rng)
    n = len(row) - 1
    ncols = max(n, int(col.max()) + 1)
    v32 = val.astype(np.float32)
    X32 = rng.uniform(-1, 1, (ncols, k)).astype(np.float32)
    A = E.Matrix(row, col, v32, ncols=ncols, fmt="K1", vtype="f32")
    Y = A.spmm(torch.from_numpy(X32).cuda()).cpu().numpy()
    _fp32_bound_ok(Y, v32.astype(np.float64), X32.astype(np.float64), row, col, port)
    # the single-RHS FP32 product of the first column, same bound
    y = A.spmv(torch.from_numpy(np.ascontiguousarray(X32[:, 0])).cuda()).cpu().numpy()
    _fp32_bound_ok(y[:, None], v32.astype(np.float64), X32[:, :1].astype(np.float64), row,
                   col, port)
    A.close()


@pytest.fixture(scope="module")
def batch_config():
    """The benchmark's batched configuration, converted once (FP32 K1 matrices)."""
    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import matgen

    work = matgen.banded_batch(256, seed=3)
    mats = [E.Matrix(r, c, v, ncols=len(r) - 1, fmt="K1", vtype="f32") for r, c, v, _ in work]
    yield work, mats
    for A in mats:
        A.close()


def test_batched_config_against_oracle(port, batch_config):
    """256 banded FP32 matrices, 1-32 right-hand sides (seed 3), one persistent launch
    replayed from a CUDA graph after the autotuner chose the blocking; a seeded sample of 24
    matrices, every column, against the oracle; the K1-unit path on the same sample."""
    from gpu_spmv_b200 import autotune
    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import matgen

    work, mats = batch_config
    ks = [w[3] for w in work]
    assert len(mats) == 256 and sum(len(w[1]) for w in work) > 250_000_000
    B = E.Batch(mats, ks)
    Xs = [matgen.batch_rhs(i, A.ncols, k, seed=3) for i, (A, k) in enumerate(zip(mats, ks))]
    B.make_operands(Xs)
    autotune.tune(B, reps=2)
    B.run(graph=True)
    torch.cuda.synchronize()
    assert B.status() == 0
    sample = np.random.default_rng(31).choice(256, 24, replace=False)
    worst = 0.0
    for i in sample:
        row, col, val, k = work[i]
        Y = B.results()[i].cpu().numpy()
        worst = max(worst, _fp32_bound_ok(Y, val.astype(np.float32).astype(np.float64),
                                          Xs[i].astype(np.float64), row, col, port))
    assert worst <= 1e-6, worst
    # the same batch on K1 units (gathers through L1 / L2): same bound
    B.set_paths(["k1"] * 256)
    for y in B.Y:
        y.fill_(float("nan"))
    B.run(graph=False)
    torch.cuda.synchronize()
    for i in sample[:8]:
        row, col, val, k = work[i]
        _fp32_bound_ok(B.results()[i].cpu().numpy(), val.astype(np.float32).astype(np.float64),
                       Xs[i].astype(np.float64), row, col, port)
    B.close()


def _transpose(row, col, val, ncols):
    n = len(row) - 1
    rows = np.repeat(np.arange(n, dtype=np.uint32), np.diff(row))
    order = np.argsort(col, kind="stable")
    rowT = np.zeros(ncols + 1, np.uint32)
    rowT[1:] = np.cumsum(np.bincount(col, minlength=ncols))
    return rowT, rows[order].astype(np.uint32), val[order]


@pytest.fixture(scope="module")
def diff_config():
    from gpu_spmv_b200 import matgen

    row, col, val = matgen.powerlaw(nrows=1048576, nnz=16777216, seed=4)
    v32 = val.astype(np.float32)
    rng = np.random.default_rng(4)
    X = rng.standard_normal((1048576, 8)).astype(np.float32)
    B = rng.standard_normal((1048576, 8)).astype(np.float32)
    return row, col, v32, X, B


def test_differentiable_config_fp32_gradients(port, diff_config):
    """y = A(v) X, loss 0.5 ||y - B||_F^2, FP32 values and 8 right-hand sides on the
    power-law matrix of 1,048,576 rows / 16.8M nnz: Xbar = A^T Ybar (both adjoint modes)
    against the oracle's CPU loop on the explicit transpose, and vbar_e = Ybar[row_e] . X[col_e]
    against its definition, each within the FP32 bound."""
    from gpu_spmv_b200 import autograd as G

    row, col, v32, X, B = diff_config
    n, k = len(row) - 1, X.shape[1]
    assert len(col) == 16777216
    op = G.SparseOperator(row, col, v32, ncols=n, vtype="f32")
    Xd = torch.from_numpy(X).cuda()
    Bd = torch.from_numpy(B).cuda()
    Y = op.mat.spmm(Xd)
    _fp32_bound_ok(Y[:, :2].cpu().numpy(), v32.astype(np.float64), X[:, :2].astype(np.float64),
                   row, col, port)
    Ybar = (Y - Bd).contiguous()
    Yb = Ybar.cpu().numpy().astype(np.float64)
    rowT, colT, valT = _transpose(row, col, v32.astype(np.float64), n)
    lensT = np.diff(rowT).astype(np.float64)
    refT = port.csr_spmm(rowT, colT, valT, Yb)
    magT = port.csr_spmm(rowT, colT, np.abs(valT), np.abs(Yb))
    for mode in ("deterministic", "atomic"):
        Xbar, vbar = op.mat.adjoint(Ybar, Xd, mode=mode)
        err = np.abs(Xbar.cpu().numpy().astype(np.float64) - refT)
        assert np.all(err <= U * (3.0 + lensT)[:, None] * magT + 1e-300), \
            (mode, float(np.max(err / np.maximum(magT, 1e-300))))
        rows = np.repeat(np.arange(n), np.diff(row))
        e = np.random.default_rng(5).choice(len(col), 200000, replace=False)
        vref = np.einsum("ek,ek->e", Yb[rows[e]], X[col[e]].astype(np.float64))
        vmag = np.einsum("ek,ek->e", np.abs(Yb[rows[e]]), np.abs(X[col[e]]).astype(np.float64))
        verr = np.abs(vbar.cpu().numpy()[e].astype(np.float64) - vref)
        assert np.all(verr <= U * (k + 3) * vmag + 1e-300), mode
    op.close()


def test_differentiable_config_central_differences(port, diff_config):
    """The same configuration in FP64 (the FP32 values and right-hand sides, widened):
    dL/dv and dL/dX from the hand-written adjoint against central differences on 64 random
    entries (32 values, 32 of X) to 1e-6, and X.grad against the explicit-transpose CSR
    gradient A^T (A X - B).  L is quadratic in each entry, so the central difference is exact
    up to rounding; it is formed from the rows the step changes (all other rows give the
    same bits in both products), so the large loss does not cancel away its digits."""
    from gpu_spmv_b200 import autograd as G

    row, col, v32, X32, B32 = diff_config
    n, k = len(row) - 1, X32.shape[1]
    val = v32.astype(np.float64)
    op = G.SparseOperator(row, col, val, ncols=n)
    v = torch.from_numpy(val).cuda().requires_grad_(True)
    X = torch.from_numpy(X32.astype(np.float64)).cuda().requires_grad_(True)
    Bd = torch.from_numpy(B32.astype(np.float64)).cuda()
    L = 0.5 * ((G.spmm(v, X, op) - Bd) ** 2).sum()
    L.backward()
    gv, gX = v.grad.clone(), X.grad.clone()
    with torch.no_grad():
        Ybar = (G.spmm(v, X, op) - Bd).cpu().numpy()
    rowT, colT, valT = _transpose(row, col, val, n)
    refT = port.csr_spmm(rowT, colT, valT, Ybar)
    magT = port.csr_spmm(rowT, colT, np.abs(valT), np.abs(Ybar))
    assert np.all(np.abs(gX.cpu().numpy() - refT) <= 1e-13 * magT + 1e-300)

    def dloss(Yp, Ym):
        # L(+) - L(-) = sum 0.5 (Y+ - Y-) (Y+ + Y- - 2B): rows the step leaves alone give 0
        return float((0.5 * (Yp - Ym) * (Yp + Ym - 2.0 * Bd)).sum())

    h = 1e-3
    rng = np.random.default_rng(64)
    with torch.no_grad():
        for idx in rng.choice(len(col), 32, replace=False):
            vp, vm = v.detach().clone(), v.detach().clone()
            vp[idx] += h
            vm[idx] -= h
            fd = dloss(G.spmm(vp, X, op), G.spmm(vm, X, op)) / (2 * h)
            g = gv[idx].item()
            assert abs(g - fd) <= 1e-6 * max(1.0, abs(g)), (int(idx), g, fd)
        Xd = X.detach()
        for flat in rng.choice(n * k, 32, replace=False):
            i, r = divmod(int(flat), k)
            Xp, Xm = Xd.clone(), Xd.clone()
            Xp[i, r] += h
            Xm[i, r] -= h
            fd = dloss(G.spmm(v.detach(), Xp, op), G.spmm(v.detach(), Xm, op)) / (2 * h)
            g = gX[i, r].item()
            assert abs(g - fd) <= 1e-6 * max(1.0, abs(g)), (i, r, g, fd)
    op.close()
