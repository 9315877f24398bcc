"""Multi-RHS K1 products and the hand-written adjoint of Y = A(v) X.

Checks: every column of the FP64 multi-RHS product equals the single-RHS K1 product bit
for bit; Xbar = A^T Ybar against the reference's CPU CSR loop applied to the explicit
transpose (per-column bound 1e-13 (|A^T||Ybar|)_j); vbar against its definition; both
adjoint modes; central finite differences of 0.5 ||A(v) X - B||^2 in FP64 on 64 random
entries (values and X) to 1e-6."""
import numpy as np
import pytest
import torch

from mats import case, csr_from_lengths, within_bound

pytestmark = pytest.mark.gpu


def _case(name, rng):
    if name == "dense_col":  # column 5 holds 2000 entries: the transpose has a split chunk
        n = 3000
        lens = rng.integers(0, 6, n)
        row, col, val = csr_from_lengths(lens, n, rng)
        r2, c2, v2 = [0], [], []
        for r in range(n):
            cs = set(col[row[r]:row[r + 1]].tolist())
            if r < 2000:
                cs.add(5)
            cs = sorted(cs)
            c2 += cs
            v2 += rng.standard_normal(len(cs)).tolist()
            r2.append(len(c2))
        return np.array(r2, np.uint32), np.array(c2, np.uint32), np.array(v2)
    return case(name, rng)


def _transpose(row, col, val, ncols):
    n = len(row) - 1
    rows = np.repeat(np.arange(n, dtype=np.uint32), np.diff(row))
    order = np.argsort(col, kind="stable")
    cnt = np.bincount(col, minlength=ncols)
    rowT = np.zeros(ncols + 1, np.uint32)
    rowT[1:] = np.cumsum(cnt)
    return rowT, rows[order].astype(np.uint32), val[order], order


CASES = ["mixed", "row0_empty", "dense_row", "dense_col", "powerlaw_small", "laplacian"]


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("k", [1, 2, 4, 8, 16, 32])
def test_spmm_columns_equal_spmv(port, name, k):
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(sum(map(ord, name)) + k)
    row, col, val = _case(name, rng)
    n = len(row) - 1
    ncols = max(n, int(col.max()) + 1)
    A = E.Matrix(row, col, val, ncols=ncols, fmt="K1")
    X = torch.from_numpy(rng.uniform(-1, 1, (ncols, k))).cuda()
    Y = A.spmm(X)
    for r in range(k):
        y = A.spmv(X[:, r].contiguous())
        assert torch.equal(Y[:, r], y), r
    xh = X[:, 0].cpu().numpy()
    _, mag = port.csr_truth(row, col, val, xh)
    assert within_bound(Y[:, 0].cpu().numpy(), port.csr_spmv(row, col, val, xh), mag)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("k", [1, 8, 32])
def test_adjoint_against_explicit_transpose(port, name, k):
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(sum(map(ord, name)) + 100 + k)
    row, col, val = _case(name, rng)
    n = len(row) - 1
    ncols = max(n, int(col.max()) + 1)
    A = E.Matrix(row, col, val, ncols=ncols, fmt="K1", adjoint=True)
    Xh = rng.uniform(-1, 1, (ncols, k))
    Yb = rng.standard_normal((n, k))
    X = torch.from_numpy(Xh).cuda()
    Ybar = torch.from_numpy(Yb).cuda()
    Xbar, vbar = A.adjoint(Ybar, X, mode="deterministic")
    Xbar2, vbar2 = A.adjoint(Ybar, X, mode="deterministic")
    assert torch.equal(Xbar, Xbar2) and torch.equal(vbar, vbar2)  # reproducible
    Xa, va = A.adjoint(Ybar, X, mode="atomic")
    assert torch.equal(va, vbar)  # same products, same order per element
    Xa0, va0 = A.adjoint(Ybar, None, mode="atomic", want_vbar=False)  # Xbar only
    assert va0 is None
    # slot order: the same numbers, in place; padding slots zero
    Xs, vs = A.adjoint(Ybar, X, mode="deterministic", order="slots")
    assert torch.equal(Xs, Xbar) and torch.equal(A.convert_values(vs, to="csr"), vbar)
    _, vsa = A.adjoint(Ybar, X, mode="atomic", order="slots")
    assert torch.equal(vsa, vs)
    real = A.convert_values(torch.ones(A.nnz, dtype=torch.float64, device="cuda"), to="slots")
    assert torch.all(vs[real == 0] == 0) and int(real.sum()) == A.nnz
    rowT, colT, valT, _ = _transpose(row, col, val, ncols)
    Xbar, Xa, Xa0 = Xbar.cpu().numpy(), Xa.cpu().numpy(), Xa0.cpu().numpy()
    for r in range(k):
        ref = port.csr_spmv(rowT, colT, valT, Yb[:, r])
        _, mag = port.csr_truth(rowT, colT, valT, Yb[:, r])
        assert within_bound(Xbar[:, r], ref, mag), r
        # atomic adds: any order of the same terms, |error| <= len_j eps (|A^T||Ybar|)_j
        lens = np.diff(rowT).astype(np.float64)
        assert np.all(np.abs(Xa[:, r] - ref) <= (lens + 1) * 2.0 ** -52 * mag + 1e-300), r
        assert np.all(np.abs(Xa0[:, r] - ref) <= (lens + 1) * 2.0 ** -52 * mag + 1e-300), r
    rows = np.repeat(np.arange(n), np.diff(row))
    vref = np.einsum("ek,ek->e", Yb[rows], Xh[col])
    vmag = np.einsum("ek,ek->e", np.abs(Yb[rows]), np.abs(Xh[col]))
    assert np.all(np.abs(vbar.cpu().numpy() - vref) <= 1e-13 * vmag + 1e-300)


@pytest.mark.parametrize("mode,order", [("deterministic", "csr"), ("atomic", "csr"),
                                        ("deterministic", "slots")])
def test_autograd_central_differences(port, mode, order):
    """FP64: d/dv and d/dX of L = 0.5 ||A(v) X - B||_F^2 against central differences (L is
    quadratic in each entry, so the difference quotient is exact up to rounding)."""
    from gpu_spmv_b200 import autograd as G

    rng = np.random.default_rng(4)
    row, col, val = case("powerlaw_small", rng)
    n = len(row) - 1
    k = 8
    op = G.SparseOperator(row, col, val, ncols=n)
    v = torch.from_numpy(val).cuda()
    if order == "slots":
        v = op.slot_values(v)
    v.requires_grad_(True)
    X = torch.from_numpy(rng.standard_normal((n, k))).cuda().requires_grad_(True)
    B = torch.from_numpy(rng.standard_normal((n, k))).cuda()

    def loss(vv, XX):
        return 0.5 * ((G.spmm(vv, XX, op, mode, order) - B) ** 2).sum()

    L = loss(v, X)
    L.backward()
    gv, gX = v.grad.clone(), X.grad.clone()
    # X.grad against the explicit-transpose CSR gradient A^T (A X - B)
    with torch.no_grad():
        Ybar = (G.spmm(v, X, op, mode, order) - B).cpu().numpy()
    rowT, colT, valT, _ = _transpose(row, col, val, n)
    for r in range(k):
        ref = port.csr_spmv(rowT, colT, valT, Ybar[:, r])
        _, mag = port.csr_truth(rowT, colT, valT, np.abs(Ybar[:, r]))
        assert np.all(np.abs(gX[:, r].cpu().numpy() - ref) <= 1e-12 * (mag + 1.0))
    h = 1e-3
    with torch.no_grad():
        for idx in rng.choice(v.numel(), 32, replace=False):
            vp, vm = v.detach().clone(), v.detach().clone()
            vp[idx] += h
            vm[idx] -= h
            fd = (loss(vp, X).item() - loss(vm, X).item()) / (2 * h)
            g = gv[idx].item()
            assert abs(g - fd) <= 1e-6 * max(1.0, abs(g)), (idx, g, fd)
        for flat in rng.choice(n * k, 32, replace=False):
            i, r = divmod(int(flat), k)
            Xp, Xm = X.detach().clone(), X.detach().clone()
            Xp[i, r] += h
            Xm[i, r] -= h
            fd = (loss(v, Xp).item() - loss(v, Xm).item()) / (2 * h)
            g = gX[i, r].item()
            assert abs(g - fd) <= 1e-6 * max(1.0, abs(g)), (i, r, g, fd)
    op.close()


def test_set_values_and_fp32_adjoint(port):
    from gpu_spmv_b200 import autograd as G
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(9)
    row, col, val = case("dense_row", rng)
    n = len(row) - 1
    k = 8
    op = G.SparseOperator(row, col, val.astype(np.float32), ncols=n, vtype="f32")
    v2 = rng.standard_normal(len(val)).astype(np.float32)
    X = torch.from_numpy(rng.standard_normal((n, k)).astype(np.float32)).cuda()
    Y = G.spmm(torch.from_numpy(v2).cuda(), X, op)
    A2 = E.Matrix(row, col, v2, ncols=n, fmt="K1", vtype="f32")
    assert torch.equal(Y, A2.spmm(X))  # new values took effect, same kernel, same bits
    # FP32 adjoint against FP64: |err| <= (len_j + 2) 2^-24 (|A^T||Ybar|)_j
    Yb = rng.standard_normal((n, k)).astype(np.float32)
    Xbar, vbar = op.mat.adjoint(torch.from_numpy(Yb).cuda(), X)
    rowT, colT, valT, _ = _transpose(row, col, v2.astype(np.float64), n)
    lens = np.diff(rowT).astype(np.float64)
    for r in range(k):
        ref, mag = port.csr_truth(rowT, colT, valT, Yb[:, r].astype(np.float64))
        err = np.abs(Xbar[:, r].cpu().numpy().astype(np.float64) - ref)
        assert np.all(err <= (lens + 2) * 2.0 ** -24 * mag + 1e-30)
    op.close()
