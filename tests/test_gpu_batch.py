"""Batched uneven multi-RHS products (gs_batch_*): one persistent launch over many K1
matrices.  Every column of every matrix sums its products in the same order as the
single-matrix product, whatever the right-hand-side blocking, so results are compared bit
for bit with Matrix.spmm; CUDA-graph replays see new operands without a new capture."""
import numpy as np
import pytest
import torch

from mats import case

pytestmark = pytest.mark.gpu


def _mats(dtype, rng, count=10):
    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import matgen

    names = ["mixed", "row0_empty", "dense_row", "k1_empty_chunk", "single_row",
             "powerlaw_small", "laplacian"]
    out = []
    for i in range(count):
        if i < len(names):
            row, col, val = case(names[i], rng)
        else:
            n = int(rng.integers(1000, 20000))
            row, col, val = matgen.banded(n, int(rng.integers(16, 257)), 5, 60,
                                          seed=int(rng.integers(1 << 30)))
        n = len(row) - 1
        ncols = max(n, int(col.max()) + 1 if len(col) else n)
        out.append(E.Matrix(row, col, val, ncols=ncols, fmt="K1", vtype=dtype))
    return out


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_batch_equals_single_products(dtype):
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(3)
    mats = _mats(dtype, rng)
    ks = [int(k) for k in rng.integers(1, 33, len(mats))]
    tdt = torch.float64 if dtype == "f64" else torch.float32
    B = E.Batch(mats, ks)
    assert B.kpad == [1 << (k - 1).bit_length() for k in ks]
    Xs = [rng.standard_normal((A.ncols, k)) for A, k in zip(mats, ks)]
    X, Y = B.make_operands(Xs)
    ref = [A.spmm(x) for A, x in zip(mats, X)]
    B.run(graph=False)
    torch.cuda.synchronize()
    for y, r in zip(Y, ref):
        assert torch.equal(y, r)
    # any blocking: the same sums in the same order
    B.set_blocking([max(1, kp // 4) for kp in B.kpad])
    for y in Y:
        y.fill_(float("nan"))
    B.run(graph=True)
    torch.cuda.synchronize()
    for y, r in zip(Y, ref):
        assert torch.equal(y, r)
    # new right-hand sides, same captured graph
    for x in X:
        x.mul_(-2.0)
    B.run(graph=True)
    torch.cuda.synchronize()
    for y, r in zip(Y, ref):
        assert torch.equal(y, -2.0 * r)
    assert all(r.dtype == tdt for r in ref)
    B.close()


def test_autotune_keeps_results(tmp_path):
    from gpu_spmv_b200 import autotune
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(5)
    mats = _mats("f32", rng, count=12)
    ks = [32, 17, 8, 3, 1, 32, 24, 9, 16, 5, 2, 31]
    B = E.Batch(mats, ks)
    X, Y = B.make_operands([rng.standard_normal((A.ncols, k)) for A, k in zip(mats, ks)])
    B.run(graph=False)
    torch.cuda.synchronize()
    before = [y.clone() for y in Y]
    cache = tmp_path / "tune.json"
    info = autotune.tune(B, reps=3, cache_path=str(cache))
    assert cache.exists() and info["choices"]
    assert all(kp % kb == 0 for kp, kb in zip(B.kpad, B.blocking))
    B.run(graph=True)
    torch.cuda.synchronize()
    for y, r in zip(Y, before):
        assert torch.equal(y, r)
    # cached choices are reused without timing
    info2 = autotune.tune(B, reps=3, cache_path=str(cache))
    assert info2["choices"] == info["choices"] and not info2["timings"]
    B.close()


def test_batch_argument_errors():
    from gpu_spmv_b200 import GSError
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(1)
    row, col, val = case("mixed", rng)
    n = len(row) - 1
    a64 = E.Matrix(row, col, val, ncols=n, fmt="K1")
    a32 = E.Matrix(row, col, val, ncols=n, fmt="K1", vtype="f32")
    csr = E.Matrix(row, col, val, ncols=n, fmt="CSR")
    with pytest.raises(GSError, match="share one value type"):
        E.Batch([a64, a32], [1, 1])
    with pytest.raises(GSError, match="K1 matrices"):
        E.Batch([csr], [1])
    with pytest.raises(GSError, match="right-hand sides"):
        E.Batch([a64], [33])
    B = E.Batch([a64], [8])
    with pytest.raises(GSError, match="set_operands"):
        B.run()
    with pytest.raises(GSError, match="power of two"):
        B.set_blocking([3])
    B.close()


def _banded_mats(dtype, rng, count, long_rows=False):
    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import matgen

    out = []
    for i in range(count):
        n = int(rng.integers(500, 30000))
        row, col, val = matgen.banded(n, int(rng.integers(16, 257)), 5, 60,
                                      seed=int(rng.integers(1 << 30)))
        if long_rows and i == 0:  # rows past one kK1Split piece (128 elements)
            row, col, val = case("mixed", rng)
        ncols = max(len(row) - 1, int(col.max()) + 1 if len(col) else 1)
        out.append(E.Matrix(row, col, val, ncols=ncols, fmt="K1", vtype=dtype))
    return out


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_row_blocks_equal_k1_units(dtype):
    """Row blocks (X band staged in shared memory) give the K1 bits: every width, every
    blocking (contiguous X blocks by bulk copy, strided ones by plain loads)."""
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(11)
    mats = _banded_mats(dtype, rng, 9, long_rows=True)
    ks = [1, 2, 3, 5, 8, 13, 16, 31, 32]
    B = E.Batch(mats, ks)
    assert B.paths == ["band"] * len(mats)
    X, Y = B.make_operands([rng.standard_normal((A.ncols, k)) for A, k in zip(mats, ks)])
    ref = [A.spmm(x) for A, x in zip(mats, X)]
    for blocking in (B.kpad, [max(1, kp // 2) for kp in B.kpad], [1] * len(mats)):
        B.set_blocking(blocking)
        for graph in (False, True):
            for y in Y:
                y.fill_(float("nan"))
            B.run(graph=graph)
            torch.cuda.synchronize()
            for i, (y, r) in enumerate(zip(Y, ref)):
                assert torch.equal(y, r), (blocking[i], graph, i)
    assert B.status() == 0
    B.set_paths(["k1"] * len(mats))
    assert B.paths == ["k1"] * len(mats)
    for y in Y:
        y.fill_(float("nan"))
    B.run()
    torch.cuda.synchronize()
    for y, r in zip(Y, ref):
        assert torch.equal(y, r)
    B.close()


def test_mixed_paths_and_refusal():
    """A matrix whose row reaches too wide a band runs as K1 units under "auto" and is
    refused under "band"; a mixed batch (both kernels) still gives the K1 bits."""
    from gpu_spmv_b200 import GSError
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(12)
    n = 60000
    row = np.array([0, 2] + [2] * (n - 1), np.uint32)
    col = np.array([0, n - 1], np.uint32)
    wide = E.Matrix(row, col, np.array([1.5, -2.0]), ncols=n, fmt="K1", vtype="f32")
    mats = [wide] + _banded_mats("f32", rng, 3)
    ks = [32, 32, 7, 1]
    B = E.Batch(mats, ks)
    assert B.paths == ["k1", "band", "band", "band"]
    X, Y = B.make_operands([rng.standard_normal((A.ncols, k)) for A, k in zip(mats, ks)])
    ref = [A.spmm(x) for A, x in zip(mats, X)]
    B.run()
    torch.cuda.synchronize()
    for y, r in zip(Y, ref):
        assert torch.equal(y, r)
    with pytest.raises(GSError, match="shared memory"):
        B.set_paths(["band"] * 4)
    assert B.paths == ["k1", "band", "band", "band"]  # unchanged after the refusal
    B.set_paths(["auto", "auto", "k1", "band"])
    assert B.paths == ["k1", "band", "k1", "band"]
    for y in Y:
        y.fill_(float("nan"))
    B.run()
    torch.cuda.synchronize()
    for y, r in zip(Y, ref):
        assert torch.equal(y, r)
    assert B.status() == 0
    B.close()


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_row_blocks_edge_matrices(dtype):
    """Row blocks on edge shapes: no stored element, one row, one column, runs of empty
    rows, rows past several kK1Split pieces and past a block's row limit; same bits as
    the single-matrix product, empty rows written as zero."""
    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200 import matgen

    from mats import csr_from_lengths

    rng = np.random.default_rng(21)
    shapes = []
    shapes.append((np.zeros(46, np.uint32), np.zeros(0, np.uint32), np.zeros(0), 45))
    shapes.append(csr_from_lengths([300], 300, rng) + (300,))
    row, col, val = csr_from_lengths(rng.integers(0, 2, 5000), 1, rng)
    shapes.append((row, col, val, 1))
    lens = rng.integers(0, 9, 9000)
    lens[100:4500] = 0
    row, col, val = csr_from_lengths(lens, 9000, rng)
    shapes.append((row, col, val, 9000))
    lens = rng.integers(1, 4, 700)
    lens[[3, 350, 699]] = [520, 257, 700]
    row, col, val = csr_from_lengths(lens, 700, rng)
    shapes.append((row, col, val, 700))
    row, col, val = matgen.banded(20000, 16, 1, 3, seed=5)  # short rows: blocks of 4096 rows
    shapes.append((row, col, val, 20000))
    mats = [E.Matrix(r, c, v, ncols=nc, fmt="K1", vtype=dtype) for r, c, v, nc in shapes]
    ks = [4, 1, 8, 1, 3, 32]  # every row with its X band fits a stage at these widths
    B = E.Batch(mats, ks)
    assert B.paths == ["band"] * len(mats)
    X, Y = B.make_operands([rng.standard_normal((A.ncols, k)) for A, k in zip(mats, ks)])
    ref = [A.spmm(x) for A, x in zip(mats, X)]
    for y in Y:
        y.fill_(float("nan"))
    B.run()
    torch.cuda.synchronize()
    for (r, _, _, _), y, rf in zip(shapes, Y, ref):
        assert torch.equal(y, rf)
        assert torch.all(y[torch.from_numpy(np.diff(r.astype(np.int64)) == 0).cuda()] == 0)
    assert B.status() == 0
    B.close()


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_row_block_height_keeps_bits(dtype):
    """Lower row-block heights cut the same matrices into more blocks and leave every sum and
    its order unchanged; out-of-range heights are refused and change nothing."""
    from gpu_spmv_b200 import GSError
    from gpu_spmv_b200 import engine as E

    rng = np.random.default_rng(17)
    mats = _banded_mats(dtype, rng, 6, long_rows=True)
    ks = [1, 4, 8, 16, 32, 3]
    B = E.Batch(mats, ks)
    X, Y = B.make_operands([rng.standard_normal((A.ncols, k)) for A, k in zip(mats, ks)])
    ref = [A.spmm(x) for A, x in zip(mats, X)]
    assert [h for h, _ in B.row_blocks] == [4096] * 6
    blocks0 = [b for _, b in B.row_blocks]
    for height in (1024, 256, 32):
        B.set_row_blocks([height] * 6)
        hb = B.row_blocks
        assert [h for h, _ in hb] == [height] * 6
        assert all(b >= b0 for (_, b), b0 in zip(hb, blocks0))
        for graph in (False, True):
            for y in Y:
                y.fill_(float("nan"))
            B.run(graph=graph)
            torch.cuda.synchronize()
            for y, r in zip(Y, ref):
                assert torch.equal(y, r), height
    assert sum(b for _, b in B.row_blocks) > sum(blocks0)
    with pytest.raises(GSError, match="rows per block"):
        B.set_row_blocks([16] * 6)
    assert [h for h, _ in B.row_blocks] == [32] * 6
    assert B.status() == 0
    B.close()
