"""Row-partitioned distributed SpMV (gpu_spmv_b200.distributed).

CPU: the nnz-balanced partition, and two gloo ranks (spawned processes) running the
all-gather / reduce-scatter exchange with the oracle as each rank's local product, checked
against the single-process product.  GPU: one NCCL rank running the engine's kernels."""
import os
import socket

import numpy as np
import pytest
import torch

from mats import case


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_nnz_balanced_rows():
    from gpu_spmv_b200.distributed import nnz_balanced_rows

    rng = np.random.default_rng(0)
    for name in ("mixed", "dense_row", "powerlaw_small", "row0_empty"):
        row, _, _ = case(name, rng)
        n, nnz = len(row) - 1, int(row[-1])
        maxlen = int(np.diff(row).max())
        for parts in (1, 2, 3, 8):
            b = nnz_balanced_rows(row, parts)
            assert b[0] == 0 and b[-1] == n and len(b) == parts + 1
            assert all(x <= y for x, y in zip(b, b[1:]))
            for k in range(parts):
                got = int(row[b[k + 1]] - row[b[k]])
                assert abs(got - nnz / parts) <= maxlen + 1


class OracleLocal:
    """A rank's local operator computed by the oracle (CPU test stand-in for the engine)."""

    def __init__(self, row, col, val, ncols, device, adjoint):
        from oracle.oracle import Port

        self.port = Port()
        self.row, self.col, self.val, self.ncols = row, col, val, ncols

    def spmv(self, x):
        return torch.from_numpy(self.port.csr_spmv(self.row, self.col, self.val, x.numpy()))

    def spmm(self, X):
        return torch.stack([self.spmv(X[:, r].contiguous()) for r in range(X.shape[1])], 1)

    def adjoint(self, Ybar, X=None, want_vbar=False):
        n = len(self.row) - 1
        rows = np.repeat(np.arange(n), np.diff(self.row))
        out = np.zeros(self.ncols)
        np.add.at(out, self.col, self.val * Ybar.numpy()[rows])
        return torch.from_numpy(out), None


def _rank_main(rank, world, port, name, seed):
    import torch.distributed as dist

    from gpu_spmv_b200.distributed import DistSpMV

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        rng = np.random.default_rng(seed)
        row, col, val = case(name, rng)
        n = len(row) - 1
        x = rng.uniform(-1, 1, n)
        yb = rng.standard_normal(n)
        D = DistSpMV(row, col, val, n, device="cpu", local_factory=OracleLocal)
        y_local = D.spmv(torch.from_numpy(x[D.r0:D.r1].copy()))
        from oracle.oracle import Port

        P = Port()
        y_ref = P.csr_spmv(row, col, val, x)
        assert np.array_equal(y_local.numpy(), y_ref[D.r0:D.r1])  # same local loop
        xb = D.adjoint(torch.from_numpy(yb[D.r0:D.r1].copy())).numpy()
        rows = np.repeat(np.arange(n), np.diff(row))
        xb_ref = np.zeros(n)
        np.add.at(xb_ref, col, val * yb[rows])
        mag = np.zeros(n)
        np.add.at(mag, col, np.abs(val * yb[rows]))
        assert np.all(np.abs(xb - xb_ref[D.r0:D.r1]) <= 1e-13 * mag[D.r0:D.r1] + 1e-300)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["mixed", "powerlaw_small"])
def test_gloo_two_ranks(name):
    import torch.multiprocessing as mp

    mp.spawn(_rank_main, args=(2, _free_port(), name, 11), nprocs=2, join=True)


class FailingLocal:
    """A local operator that cannot be built (a rank whose block fails)."""

    def __init__(self, *args):
        raise RuntimeError("this rank's block could not be built")


def _bench_rank_main(rank, world, port, fail_rank):
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        rng = np.random.default_rng(5)
        row, col, val = case("powerlaw_small", rng)
        n = len(row) - 1
        x = rng.uniform(-1, 1, n)
        factory = FailingLocal if rank == fail_rank else OracleLocal
        out = bench.time_dist(row, col, val, x, 3, 1, "cpu", local_factory=factory)
        if fail_rank >= 0:
            assert set(out) == {"error"}, out
            if rank == fail_rank:
                assert "could not be built" in out["error"]
        else:
            assert "error" not in out, out
            assert out["ranks"] == world and sum(out["rows_per_rank"]) == n
            assert sum(out["nnz_per_rank"]) == len(col)
            assert out["us_per_product"] > 0 and out["scaling"] == "strong"
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("fail_rank", [-1, 1], ids=["both_build", "rank1_fails"])
def test_bench_dist_two_ranks(fail_rank):
    """bench.time_dist over two gloo ranks: the shared matrix's row blocks cover it, the time
    is reported; a rank that cannot build its block makes every rank return the error
    instead of entering the timed all-gathers alone."""
    import torch.multiprocessing as mp

    mp.spawn(_bench_rank_main, args=(2, _free_port(), fail_rank), nprocs=2, join=True)


@pytest.mark.gpu
def test_bench_dist_one_nccl_rank():
    """bench.time_dist on one NCCL rank with the engine's K1 block on the GPU."""
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0,
                            world_size=1, device_id=torch.device("cuda", 0))
    try:
        rng = np.random.default_rng(3)
        row, col, val = case("powerlaw_small", rng)
        n = len(row) - 1
        out = bench.time_dist(row, col, val, rng.uniform(-1, 1, n), 5, 2,
                              torch.device("cuda", 0))
        assert "error" not in out, out
        assert out["rows_per_rank"] == [n] and out["gflops"] > 0
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_nccl_one_rank_engine(port):
    import torch.distributed as dist

    from gpu_spmv_b200 import engine as E
    from gpu_spmv_b200.distributed import DistSpMV

    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{_free_port()}", rank=0,
                            world_size=1, device_id=torch.device("cuda", 0))
    try:
        rng = np.random.default_rng(2)
        row, col, val = case("powerlaw_small", rng)
        n = len(row) - 1
        D = DistSpMV(row, col, val, n, adjoint=True)
        A = E.Matrix(row, col, val, ncols=n, fmt="K1", adjoint=True)
        x = torch.from_numpy(rng.uniform(-1, 1, n)).cuda()
        assert torch.equal(D.spmv(x), A.spmv(x))
        X = torch.from_numpy(rng.uniform(-1, 1, (n, 8))).cuda()
        assert torch.equal(D.spmv(X), A.spmm(X))
        yb = torch.from_numpy(rng.standard_normal(n)).cuda()
        assert torch.equal(D.adjoint(yb), A.adjoint(yb, None, want_vbar=False)[0])
    finally:
        dist.destroy_process_group()
