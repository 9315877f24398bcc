"""The seeded workload generators: exact sizes of the benchmark configurations, structural
invariants (sorted distinct columns, bounds), determinism, and the stencil/Laplacian
values."""
import numpy as np

from gpu_spmv_b200 import matgen


def _rows_strictly_increasing(row, col):
    starts = np.zeros(len(col), bool)
    nz = np.diff(row) > 0
    starts[row[:-1][nz]] = True
    d = np.diff(col.astype(np.int64))
    return bool(np.all(d[~starts[1:]] > 0))


def test_laplacian_512():
    row, col, val = matgen.laplacian2d(512)
    assert len(row) - 1 == 262144 and len(col) == 1308672
    assert _rows_strictly_increasing(row, col)
    lens = np.diff(row)
    assert sorted(np.unique(lens).tolist()) == [3, 4, 5]
    assert np.count_nonzero(lens == 3) == 4 and np.count_nonzero(lens == 4) == 2040
    diag = val[np.repeat(np.arange(262144), lens) == col]
    assert np.all(diag == 4.0) and np.all(val[val != 4.0] == -1.0)


def test_powerlaw_small_properties():
    row, col, val = matgen.powerlaw(nrows=100000, nnz=1600000, max_len=2000, seed=5)
    lens = np.diff(row)
    assert lens.sum() == 1600000 and lens.min() >= 1 and lens.max() <= 2000
    assert _rows_strictly_increasing(row, col)
    assert col.max() < 100000
    r2, c2, v2 = matgen.powerlaw(nrows=100000, nnz=1600000, max_len=2000, seed=5)
    assert np.array_equal(row, r2) and np.array_equal(col, c2) and np.array_equal(val, v2)
    r3, _, _ = matgen.powerlaw(nrows=100000, nnz=1600000, max_len=2000, seed=6)
    assert not np.array_equal(row, r3)
    assert abs(val.mean()) < 0.01 and abs(val.std() - 1) < 0.01


def test_stencil27_small():
    row, col, val = matgen.stencil27(10, seed=2)
    assert len(row) - 1 == 1000 and len(col) == 28 ** 3
    assert _rows_strictly_increasing(row, col)
    n = 1000
    diag = np.repeat(np.arange(n), np.diff(row)) == col
    assert np.all(val[diag] == 26.0)
    off = val[~diag]
    assert off.min() >= -1.1 and off.max() <= -0.9


def test_banded_in_band():
    row, col, val = matgen.banded(5000, 40, 5, 60, seed=3)
    lens = np.diff(row)
    assert lens.min() >= 5 and lens.max() <= 60
    r = np.repeat(np.arange(5000), lens)
    assert np.all(np.abs(col.astype(np.int64) - r) <= 40)
    assert _rows_strictly_increasing(row, col)


def test_vector_seeded():
    a = matgen.vector(1000, "uniform", -1, 1, seed=0)
    b = matgen.vector(1000, "uniform", -1, 1, seed=0)
    assert np.array_equal(a, b) and a.min() >= -1 and a.max() < 1
    z = matgen.vector(100000, "normal", seed=4)
    assert abs(z.mean()) < 0.02 and abs(z.std() - 1) < 0.02


def test_reference_arm_generator_same_bytes():
    """The reference arm of bench.py builds its inputs with oracle/_build/libgs_workload.so
    (the same generator source built apart from the engine library): the same seed must give
    the same bytes as the engine's generator, for the headline power-law configuration
    (4,194,304 rows, 67,108,864 nnz, seed 1, x seed 1001) and the other workloads."""
    from oracle import workload as W

    for a, b in ((matgen.powerlaw(seed=1), W.powerlaw(seed=1)),
                 (matgen.stencil27(40, seed=2), W.stencil27(40, seed=2)),
                 (matgen.laplacian2d(64), W.laplacian2d(64)),
                 (matgen.banded(3000, 100, 5, 60, seed=3001), W.banded(3000, 100, 5, 60, seed=3001))):
        for u, v in zip(a, b):
            assert u.dtype == v.dtype and np.array_equal(u.view(np.uint8), v.view(np.uint8))
    for dist, seed in (("uniform", 1001), ("normal", 2)):
        u = matgen.vector(4194304, dist, -1.0, 1.0, seed=seed)
        v = W.vector(4194304, dist, -1.0, 1.0, seed=seed)
        assert np.array_equal(u.view(np.uint8), v.view(np.uint8))
